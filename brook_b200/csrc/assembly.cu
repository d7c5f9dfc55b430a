// Device assembly of packed skeletons. Every path vertex becomes one 64-bit key
// (skeleton, x, y, z) — skeleton in the high bits, then x, y, z, so that one stable radix sort
// orders every skeleton's vertices by (x, y, z) exactly as consolidate's lexicographic sort does.
// Runs of equal keys collapse to one vertex (its radius from the first occurrence); consecutive
// path vertices give edges as (lower, higher) pairs of global vertex indices, which one more
// radix sort orders per skeleton; duplicates and vertices on no edge drop out by flag scans.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <string>
#include <stdexcept>

#include "assembly.hpp"

namespace bk {
namespace {

constexpr unsigned long long kNoEdge = ~0ull;

struct KeyLayout {
  int bz, by, bx, shift;  // bit widths of z, y, x; shift = bx + by + bz
};

__global__ void occurrence_keys(const int *store, const float *dbf, const int *src, const int *len, const int *group,
                                const int *volume, const long long *occ_begin, const long long *arena_offset,
                                const int *arena_dims, const int *arena_origin, KeyLayout k, unsigned long long *keys,
                                int *index, float *radius, unsigned char *first) {
  const int p = blockIdx.x;
  const int n = len[p], vol = volume[p];
  const long long base = occ_begin[p];
  const int sx = arena_dims[3 * vol], sy = arena_dims[3 * vol + 1];
  const int ox = arena_origin[3 * vol], oy = arena_origin[3 * vol + 1], oz = arena_origin[3 * vol + 2];
  const unsigned long long g = static_cast<unsigned long long>(group[p]) << k.shift;
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const int v = store[src[p] + q];
    long long r = v - arena_offset[vol];
    const int z = int(r / ((long long)sx * sy));
    r -= (long long)z * sx * sy;
    const int y = int(r / sx) + oy, x = int(r - (long long)(y - oy) * sx) + ox;
    const long long o = base + q;
    keys[o] = g | (static_cast<unsigned long long>(x) << (k.by + k.bz)) | (static_cast<unsigned long long>(y) << k.bz) |
              static_cast<unsigned long long>(z + oz);
    index[o] = int(o);
    radius[o] = dbf[v];
    first[o] = q == 0;
  }
}

__global__ void run_heads(const unsigned long long *sorted, int *head, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) head[i] = (i == 0 || sorted[i] != sorted[i - 1]) ? 1 : 0;
}

// inverse[occurrence] = its unique vertex; the run head writes the vertex's key and radius
__global__ void unique_vertices(const unsigned long long *sorted, const int *order, const int *head, const int *rank,
                                const float *radius, long long n, int *inverse, unsigned long long *ukey, float *urad) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int u = rank[i] + head[i] - 1;
  const int o = order[i];
  inverse[o] = u;
  if (head[i]) {
    ukey[u] = sorted[i];
    urad[u] = radius[o];
  }
}

__global__ void edge_keys(const int *inverse, const unsigned char *first, long long n, unsigned long long *keys) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long key = kNoEdge;
  if (!first[i]) {
    unsigned a = unsigned(inverse[i - 1]), b = unsigned(inverse[i]);
    if (a > b) { const unsigned t = a; a = b; b = t; }
    if (a != b) key = (static_cast<unsigned long long>(a) << 32) | b;
  }
  keys[i] = key;
}

__global__ void edge_heads(const unsigned long long *sorted, int *head, unsigned char *used, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long e = sorted[i];
  const int h = e != kNoEdge && (i == 0 || e != sorted[i - 1]);
  head[i] = h;
  if (h) {
    used[unsigned(e >> 32)] = 1;
    used[unsigned(e)] = 1;
  }
}

__global__ void widen(const unsigned char *in, int *out, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

__global__ void vertex_out(const unsigned long long *ukey, const float *urad, const int *used, const int *rank,
                           long long n, KeyLayout k, float ax, float ay, float az, float *vertices, float *radii,
                           int *vcount) {
  const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n || !used[u]) return;
  const unsigned long long key = ukey[u];
  const int j = rank[u];
  const int z = int(key & ((1ull << k.bz) - 1));
  const int y = int((key >> k.bz) & ((1ull << k.by) - 1));
  const int x = int((key >> (k.by + k.bz)) & ((1ull << k.bx) - 1));
  vertices[3LL * j] = __fmul_rn(float(x), ax);
  vertices[3LL * j + 1] = __fmul_rn(float(y), ay);
  vertices[3LL * j + 2] = __fmul_rn(float(z), az);
  radii[j] = urad[u];
  atomicAdd(vcount + int(key >> k.shift), 1);
}

__global__ void edge_count(const unsigned long long *sorted, const int *head, const unsigned long long *ukey,
                           long long n, int shift, int *ecount) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && head[i]) atomicAdd(ecount + int(ukey[unsigned(sorted[i] >> 32)] >> shift), 1);
}

// local edges: global vertex ranks minus the skeleton's first vertex
__global__ void edge_out(const unsigned long long *sorted, const int *head, const int *erank, const int *vrank,
                         const unsigned long long *ukey, const long long *vbase, long long n, int shift,
                         uint32_t *edges) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !head[i]) return;
  const unsigned a = unsigned(sorted[i] >> 32), b = unsigned(sorted[i]);
  const long long base = vbase[int(ukey[a] >> shift)];
  const int j = erank[i];
  edges[2LL * j] = uint32_t(vrank[a] - base);
  edges[2LL * j + 1] = uint32_t(vrank[b] - base);
}

int bits_for(long long count) {  // bits to hold 0 .. count - 1
  int b = 1;
  while ((1LL << b) < count) ++b;
  return b;
}

template <class T>
void exclusive_sum(Context &ctx, const T *in, T *out, long long n) {
  size_t temp = 0;
  BK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, in, out, (int)n, ctx.stream()));
  Buffer<unsigned char> scratch(ctx, temp);
  BK_CUDA(cub::DeviceScan::ExclusiveSum(scratch.data(), temp, in, out, (int)n, ctx.stream()));
}

}  // namespace

AssemblyResult assemble(Context &ctx, const int *store, const float *dbf, const AssemblyPaths &paths,
                        const std::vector<long long> &arena_offset, const std::vector<std::array<int, 3>> &arena_dims,
                        const std::vector<std::array<int, 3>> &arena_origin, const float anisotropy[3]) {
  cudaStream_t s = ctx.stream();
  auto host_t = std::chrono::steady_clock::now();
  auto host_mark = [&](const char *step) {  // host time of each step: ctx.stats["host_ms_assemble_<step>"]
    const auto now = std::chrono::steady_clock::now();
    ctx.stats[std::string("host_ms_assemble_") + step] += std::chrono::duration<double, std::milli>(now - host_t).count();
    host_t = now;
  };
  AssemblyResult out;
  const int G = paths.groups, npaths = int(paths.src.size());
  out.vertex_offsets.assign(G + 1, 0);
  out.edge_offsets.assign(G + 1, 0);
  std::vector<long long> occ_begin(npaths + 1, 0);
  for (int p = 0; p < npaths; ++p) occ_begin[p + 1] = occ_begin[p] + paths.len[p];
  const long long P = occ_begin[npaths];
  if (G == 0 || P == 0) return out;
  if (P >= (1LL << 31)) throw std::invalid_argument("too many path vertices");
  KeyLayout k{};
  int mx = 1, my = 1, mz = 1;
  for (size_t r = 0; r < arena_dims.size(); ++r) {
    const auto &d = arena_dims[r], &o = arena_origin[r];
    mx = std::max(mx, d[0] + o[0]); my = std::max(my, d[1] + o[1]); mz = std::max(mz, d[2] + o[2]);
  }
  k.bx = bits_for(mx); k.by = bits_for(my); k.bz = bits_for(mz);
  k.shift = k.bx + k.by + k.bz;
  const int end_bit = k.shift + bits_for(G);
  if (end_bit > 64) throw std::invalid_argument("skeleton keys exceed 64 bits");

  std::vector<int> dims_flat, origin_flat;
  for (const auto &d : arena_dims) dims_flat.insert(dims_flat.end(), d.begin(), d.end());
  for (const auto &o : arena_origin) origin_flat.insert(origin_flat.end(), o.begin(), o.end());
  auto d_src = to_device(ctx, paths.src), d_len = to_device(ctx, paths.len), d_group = to_device(ctx, paths.group);
  auto d_volume = to_device(ctx, paths.volume);
  auto d_occ = to_device(ctx, occ_begin), d_aoff = to_device(ctx, arena_offset);
  auto d_dims = to_device(ctx, dims_flat), d_origin = to_device(ctx, origin_flat);

  host_mark("upload");
  // every occurrence: key, index, radius, first-of-path
  Buffer<unsigned long long> keys(ctx, P), sorted(ctx, P);
  Buffer<int> index(ctx, P), order(ctx, P);
  Buffer<float> radius(ctx, P);
  Buffer<unsigned char> first(ctx, P);
  host_mark("allocate");
  occurrence_keys<<<npaths, 128, 0, s>>>(store, dbf, d_src.data(), d_len.data(), d_group.data(), d_volume.data(),
                                         d_occ.data(), d_aoff.data(), d_dims.data(), d_origin.data(), k, keys.data(),
                                         index.data(), radius.data(), first.data()); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  host_mark("keys");
  size_t temp = 0;
  BK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, keys.data(), sorted.data(), index.data(), order.data(), (int)P,
                                          0, end_bit, s));
  host_mark("sort_query");
  {
    Buffer<unsigned char> scratch(ctx, temp);
    host_mark("sort_scratch");
    BK_CUDA(cub::DeviceRadixSort::SortPairs(scratch.data(), temp, keys.data(), sorted.data(), index.data(),
                                            order.data(), (int)P, 0, end_bit, s));
  }
  host_mark("sort");
  // unique vertices (stable sort: a run's head is the earliest occurrence)
  Buffer<int> head(ctx, P), rank(ctx, P), inverse(ctx, P);
  run_heads<<<blocks_for(P), 256, 0, s>>>(sorted.data(), head.data(), P); ++ctx.launches;
  exclusive_sum(ctx, head.data(), rank.data(), P);
  Buffer<unsigned long long> ukey(ctx, P);
  Buffer<float> urad(ctx, P);
  unique_vertices<<<blocks_for(P), 256, 0, s>>>(sorted.data(), order.data(), head.data(), rank.data(), radius.data(), P,
                                                inverse.data(), ukey.data(), urad.data()); ++ctx.launches;
  // edges between consecutive path vertices, sorted and unique
  edge_keys<<<blocks_for(P), 256, 0, s>>>(inverse.data(), first.data(), P, keys.data()); ++ctx.launches;
  temp = 0;
  BK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, temp, keys.data(), sorted.data(), (int)P, 0, 64, s));
  {
    Buffer<unsigned char> scratch(ctx, temp);
    BK_CUDA(cub::DeviceRadixSort::SortKeys(scratch.data(), temp, keys.data(), sorted.data(), (int)P, 0, 64, s));
  }
  Buffer<unsigned char> used8(ctx, P);
  used8.zero();
  edge_heads<<<blocks_for(P), 256, 0, s>>>(sorted.data(), head.data(), used8.data(), P); ++ctx.launches;
  Buffer<int> erank(ctx, P), used(ctx, P), vrank(ctx, P);
  exclusive_sum(ctx, head.data(), erank.data(), P);
  widen<<<blocks_for(P), 256, 0, s>>>(used8.data(), used.data(), P); ++ctx.launches;
  exclusive_sum(ctx, used.data(), vrank.data(), P);
  BK_CUDA(cudaGetLastError());
  const auto tail = [&](const Buffer<int> &flag, const Buffer<int> &r) {
    int a = 0, b = 0;
    BK_CUDA(cudaMemcpyAsync(&a, flag.data() + P - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    BK_CUDA(cudaMemcpyAsync(&b, r.data() + P - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    ctx.synchronize();
    return (long long)a + b;
  };
  host_mark("queue");
  const long long V = tail(used, vrank), E = tail(head, erank);
  host_mark("counts");
  // per-skeleton counts -> offsets
  Buffer<int> vcount(ctx, G), ecount(ctx, G);
  vcount.zero();
  ecount.zero();
  out.vertices = Buffer<float>(ctx, std::max(3 * V, 1LL));
  out.radii = Buffer<float>(ctx, std::max(V, 1LL));
  out.edges = Buffer<uint32_t>(ctx, std::max(2 * E, 1LL));
  vertex_out<<<blocks_for(P), 256, 0, s>>>(ukey.data(), urad.data(), used.data(), vrank.data(), P, k, anisotropy[0],
                                           anisotropy[1], anisotropy[2], out.vertices.data(), out.radii.data(),
                                           vcount.data()); ++ctx.launches;
  edge_count<<<blocks_for(P), 256, 0, s>>>(sorted.data(), head.data(), ukey.data(), P, k.shift, ecount.data());
  ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  const auto hv = vcount.download(), he = ecount.download();
  host_mark("offsets");
  for (int g = 0; g < G; ++g) {
    out.vertex_offsets[g + 1] = out.vertex_offsets[g] + hv[g];
    out.edge_offsets[g + 1] = out.edge_offsets[g] + he[g];
  }
  std::vector<long long> vbase(out.vertex_offsets.begin(), out.vertex_offsets.end() - 1);
  auto d_vbase = to_device(ctx, vbase);
  edge_out<<<blocks_for(P), 256, 0, s>>>(sorted.data(), head.data(), erank.data(), vrank.data(), ukey.data(),
                                         d_vbase.data(), P, k.shift, out.edges.data()); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  return out;
}

}  // namespace bk
