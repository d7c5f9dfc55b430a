// Merge of skeleton fragments on the device: the pieces of overlapping chunks, each placed at its
// chunk's physical origin, become one skeleton per label (the reference's merge_fragments and
// merge_parts, packed.cpp:67-86 and packed_merge.cu:88-166 of giorgioangel/brook, with its
// defaults: labels sorted ascending, labels without edges kept). Vertices of one label that land
// on the same physical point (float32 equality after adding the origin) are one vertex, whose
// radius is its first occurrence's in fragment order; edges map onto the merged vertices, self
// loops drop out, duplicates collapse, and vertices on no edge are dropped. A label's vertices come
// out sorted by (x, y, z) (-0 and +0 equal, NaN last) and its edges as sorted (lower, higher) pairs.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <map>
#include <stdexcept>

#include "merge.hpp"

namespace bk {
namespace {

struct Piece {
  const float *vertices, *radii;
  const uint32_t *edges;
  int nv, ne, vbase, ebase, group;
  float origin[3];
};

template <bool Edges>
__device__ int piece_of(const Piece *pieces, int count, int i) {
  int lo = 0, hi = count;
  while (lo + 1 < hi) {
    const int mid = lo + (hi - lo) / 2;
    const int begin = Edges ? pieces[mid].ebase : pieces[mid].vbase;
    if (begin <= i) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void gather_vertices(const Piece *pieces, int count, int n, float *vertices, float *radii, int *group,
                                int *order) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Piece &p = pieces[piece_of<false>(pieces, count, i)];
  const int local = i - p.vbase;
  for (int a = 0; a < 3; ++a) vertices[3LL * i + a] = __fadd_rn(p.vertices[3LL * local + a], p.origin[a]);
  radii[i] = p.radii[local];
  group[i] = p.group;
  order[i] = i;
}

// An order-preserving unsigned key of a float (-0 and +0 alike, NaN after everything).
__device__ __forceinline__ unsigned float_order(float v) {
  if (isnan(v)) return 0xFFFFFFFFu;
  const unsigned b = v == 0.0f ? 0u : __float_as_uint(v);
  return b ^ ((b & 0x80000000u) ? 0xFFFFFFFFu : 0x80000000u);
}

__global__ void axis_keys(const float *vertices, const int *group, const int *order, unsigned *keys, int n, int axis) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = order[i];
  keys[i] = axis < 3 ? float_order(vertices[3LL * v + axis]) : unsigned(group[v]);
}

// 1 where sorted position i starts a new vertex (another group or another point).
struct NewPoint {
  const float *vertices;
  const int *group, *order;
  __device__ int operator()(int i) const {
    if (i == 0) return 1;
    const int a = order[i - 1], b = order[i];
    if (group[a] != group[b]) return 1;
    for (int k = 0; k < 3; ++k)
      if (vertices[3LL * a + k] != vertices[3LL * b + k]) return 1;
    return 0;
  }
};

__global__ void number_points(const int *order, const int *rank, int n, NewPoint is_new, int *merged, int *first) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = rank[i] - 1;
  merged[order[i]] = r;
  if (is_new(i)) first[r] = order[i];
}

__global__ void edge_keys(const Piece *pieces, int count, int n, const int *merged, unsigned long long *keys,
                          int *error) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Piece &p = pieces[piece_of<true>(pieces, count, i)];
  const int local = i - p.ebase;
  unsigned a = p.edges[2LL * local], b = p.edges[2LL * local + 1];
  keys[i] = ~0ull;
  if (a >= unsigned(p.nv) || b >= unsigned(p.nv)) { atomicExch(error, 1); return; }
  a = unsigned(merged[p.vbase + a]);
  b = unsigned(merged[p.vbase + b]);
  if (a != b) keys[i] = (static_cast<unsigned long long>(min(a, b)) << 32) | max(a, b);
}

__global__ void mark_used(const unsigned long long *edges, int n, int *used) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) { used[edges[i] >> 32] = 1; used[unsigned(edges[i])] = 1; }
}

__global__ void write_vertices(const float *vertices, const float *radii, const int *group, const int *first,
                               const int *used, const int *rank, int n, float *out, float *out_radii, int *counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !used[i]) return;
  const int src = first[i], dst = rank[i] - 1;
  for (int k = 0; k < 3; ++k) out[3LL * dst + k] = vertices[3LL * src + k];
  out_radii[dst] = radii[src];
  atomicAdd(counts + group[src], 1);
}

__global__ void count_edges(const unsigned long long *edges, int n, const int *first, const int *group, int *counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(counts + group[first[edges[i] >> 32]], 1);
}

__global__ void write_edges(const unsigned long long *edges, int n, const int *first, const int *group, const int *rank,
                            const long long *vbase, uint32_t *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned a = unsigned(edges[i] >> 32), b = unsigned(edges[i]);
  const long long base = vbase[group[first[a]]];
  out[2LL * i] = uint32_t(rank[a] - 1 - base);
  out[2LL * i + 1] = uint32_t(rank[b] - 1 - base);
}

int last_of(Context &ctx, const Buffer<int> &values, int n) {
  return n ? values.download(1, size_t(n - 1))[0] : 0;
}

}  // namespace

Packed merge_fragments(Context &ctx, const std::vector<const Packed *> &fragments,
                       const std::vector<std::array<float, 3>> &origins) {
  if (fragments.size() != origins.size()) throw std::invalid_argument("fragment/origin count mismatch");
  cudaStream_t s = ctx.stream();
  Packed out;
  if (!fragments.empty()) out.anisotropy = fragments.front()->anisotropy;
  // labels with vertices, ascending; the group of a label is its rank
  std::map<int64_t, int> rank_of;
  for (const Packed *f : fragments)
    for (size_t k = 0; k < f->labels.size(); ++k)
      if (f->vertex_offsets[k + 1] > f->vertex_offsets[k]) rank_of[f->labels[k]] = 0;
  int g = 0;
  for (auto &kv : rank_of) { kv.second = g++; out.labels.push_back(kv.first); }
  out.device_vertices = std::make_shared<DeviceStorage>(0, ctx.device());
  out.device_edges = std::make_shared<DeviceStorage>(0, ctx.device());
  out.device_radii = std::make_shared<DeviceStorage>(0, ctx.device());
  if (out.labels.empty()) return out;
  // every fragment's arrays on the device (host fragments are uploaded), one piece per skeleton
  std::vector<Buffer<float>> up_vertices, up_radii;
  std::vector<Buffer<uint32_t>> up_edges;
  std::vector<Piece> pieces;
  long long nv = 0, ne = 0;
  for (size_t f = 0; f < fragments.size(); ++f) {
    const Packed &p = *fragments[f];
    const float *vert = nullptr, *rad = nullptr;
    const uint32_t *edg = nullptr;
    if (p.on_device()) {
      vert = static_cast<const float *>(p.device_vertices->ptr);
      rad = static_cast<const float *>(p.device_radii->ptr);
      edg = static_cast<const uint32_t *>(p.device_edges->ptr);
    } else {
      up_vertices.push_back(to_device(ctx, p.vertices));
      up_radii.push_back(to_device(ctx, p.radii));
      up_edges.push_back(to_device(ctx, p.edges));
      vert = up_vertices.back().data();
      rad = up_radii.back().data();
      edg = up_edges.back().data();
    }
    for (size_t k = 0; k < p.labels.size(); ++k) {
      const long long v0 = p.vertex_offsets[k], v1 = p.vertex_offsets[k + 1];
      const long long e0 = p.edge_offsets[k], e1 = p.edge_offsets[k + 1];
      if (v1 == v0) {
        if (e1 != e0) throw std::invalid_argument("edges without vertices");
        continue;
      }
      if (nv + (v1 - v0) >= INT32_MAX || ne + (e1 - e0) >= INT32_MAX) throw std::invalid_argument("merge too large");
      Piece pc{};
      pc.vertices = vert + 3 * v0;
      pc.radii = rad + v0;
      pc.edges = edg + 2 * e0;
      pc.nv = int(v1 - v0);
      pc.ne = int(e1 - e0);
      pc.vbase = int(nv);
      pc.ebase = int(ne);
      pc.group = rank_of.at(p.labels[k]);
      for (int a = 0; a < 3; ++a) pc.origin[a] = origins[f][a];
      pieces.push_back(pc);
      nv += pc.nv;
      ne += pc.ne;
    }
  }
  const int n = int(nv), m = int(ne), np = int(pieces.size());
  Buffer<Piece> d_pieces = to_device(ctx, pieces);
  Buffer<float> vertices(ctx, 3 * nv), radii(ctx, nv);
  Buffer<int> group(ctx, nv), order_a(ctx, nv), order_b(ctx, nv), rank(ctx, nv), merged(ctx, nv);
  Buffer<unsigned> keys_a(ctx, nv), keys_b(ctx, nv);
  Buffer<unsigned char> scratch;
  auto with_scratch = [&](auto op) {  // a CUB call with scratch sized by its own query
    size_t bytes = 0;
    BK_CUDA(op(nullptr, bytes));
    if (bytes > scratch.size()) scratch = Buffer<unsigned char>(ctx, bytes);
    BK_CUDA(op(scratch.data(), bytes));
  };
  gather_vertices<<<blocks_for(n), 256, 0, s>>>(d_pieces.data(), np, n, vertices.data(), radii.data(), group.data(),
                                                order_a.data()); ++ctx.launches;
  // stable least-significant-first sorts: z, y, x, then the group (ties keep fragment order)
  for (int axis : {2, 1, 0, 3}) {
    axis_keys<<<blocks_for(n), 256, 0, s>>>(vertices.data(), group.data(), order_a.data(), keys_a.data(), n, axis);
    ++ctx.launches;
    with_scratch([&](void *p, size_t &bytes) {
      return cub::DeviceRadixSort::SortPairs(p, bytes, keys_a.data(), keys_b.data(), order_a.data(), order_b.data(), n,
                                             0, 32, s);
    });
    std::swap(order_a, order_b);
  }
  BK_CUDA(cudaGetLastError());
  NewPoint is_new{vertices.data(), group.data(), order_a.data()};
  auto flags = thrust::make_transform_iterator(thrust::counting_iterator<int>(0), is_new);
  with_scratch([&](void *p, size_t &bytes) { return cub::DeviceScan::InclusiveSum(p, bytes, flags, rank.data(), n, s); });
  const int points = last_of(ctx, rank, n);
  Buffer<int> first(ctx, points);
  number_points<<<blocks_for(n), 256, 0, s>>>(order_a.data(), rank.data(), n, is_new, merged.data(), first.data());
  ++ctx.launches;
  // edges on the merged points: (lower, higher) keys, self loops as the all-ones key, sorted, unique
  Buffer<unsigned long long> ekeys(ctx, ne + 1), esorted(ctx, ne + 1);
  Buffer<int> error(ctx, 1), selected(ctx, 1);
  error.zero();
  if (m) {
    edge_keys<<<blocks_for(m), 256, 0, s>>>(d_pieces.data(), np, m, merged.data(), ekeys.data(), error.data());
    ++ctx.launches;
  }
  BK_CUDA(cudaMemsetAsync(ekeys.data() + ne, 0xFF, sizeof(unsigned long long), s));  // a sentinel
  with_scratch([&](void *p, size_t &bytes) {
    return cub::DeviceRadixSort::SortKeys(p, bytes, ekeys.data(), esorted.data(), m + 1, 0, 64, s);
  });
  with_scratch([&](void *p, size_t &bytes) {
    return cub::DeviceSelect::Unique(p, bytes, esorted.data(), ekeys.data(), selected.data(), m + 1, s);
  });
  const int edges = selected.download(1)[0] - 1;  // the sentinel (and the self loops) sort last
  if (error.download(1)[0]) throw std::invalid_argument("a fragment's edge is out of its vertex range");
  Buffer<int> used(ctx, points > 0 ? points : 1), vrank(ctx, points > 0 ? points : 1);
  used.zero();
  if (edges > 0) {
    mark_used<<<blocks_for(edges), 256, 0, s>>>(ekeys.data(), edges, used.data());
    ++ctx.launches;
  }
  with_scratch([&](void *p, size_t &bytes) {
    return cub::DeviceScan::InclusiveSum(p, bytes, used.data(), vrank.data(), points, s);
  });
  const int kept = last_of(ctx, vrank, points);
  const int G = int(out.labels.size());
  Buffer<int> vcount(ctx, G), ecount(ctx, G);
  vcount.zero();
  ecount.zero();
  out.device_vertices = std::make_shared<DeviceStorage>(size_t(kept) * 3 * sizeof(float), ctx.device());
  out.device_radii = std::make_shared<DeviceStorage>(size_t(kept) * sizeof(float), ctx.device());
  out.device_edges = std::make_shared<DeviceStorage>(size_t(edges > 0 ? edges : 0) * 2 * sizeof(uint32_t), ctx.device());
  if (points > 0) {
    write_vertices<<<blocks_for(points), 256, 0, s>>>(vertices.data(), radii.data(), group.data(), first.data(),
                                                      used.data(), vrank.data(), points,
                                                      static_cast<float *>(out.device_vertices->ptr),
                                                      static_cast<float *>(out.device_radii->ptr), vcount.data());
    ++ctx.launches;
  }
  if (edges > 0) {
    count_edges<<<blocks_for(edges), 256, 0, s>>>(ekeys.data(), edges, first.data(), group.data(), ecount.data());
    ++ctx.launches;
  }
  BK_CUDA(cudaGetLastError());
  const auto vc = vcount.download(), ec = ecount.download();
  std::vector<long long> vbase(G + 1, 0);
  out.vertex_offsets = {0};
  out.edge_offsets = {0};
  for (int k = 0; k < G; ++k) {
    vbase[k + 1] = vbase[k] + vc[k];
    out.vertex_offsets.push_back(out.vertex_offsets.back() + vc[k]);
    out.edge_offsets.push_back(out.edge_offsets.back() + ec[k]);
  }
  if (edges > 0) {
    Buffer<long long> d_vbase = to_device(ctx, vbase);
    write_edges<<<blocks_for(edges), 256, 0, s>>>(ekeys.data(), edges, first.data(), group.data(), vrank.data(),
                                                  d_vbase.data(), static_cast<uint32_t *>(out.device_edges->ptr));
    ++ctx.launches;
    BK_CUDA(cudaGetLastError());
  }
  ctx.synchronize();
  return out;
}

}  // namespace bk
