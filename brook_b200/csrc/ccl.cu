// Connected components on sm_100a: union-find over the 13 forward neighbours of every voxel
// (the root of a component is its lowest flat index, since links always point from the larger
// root to the smaller), a read-only flatten, and ids from an exclusive scan of the root flags in
// flat order: id k belongs to the k-th root in ascending flat order, the reference's canonical
// numbering (ccl.cu:25-63 of giorgioangel/brook) without its host sort.
//
// The union runs in two kernels: tile_union labels 32x8x8 tiles in shared memory (labels staged
// once, each x run of equal labels linked to its first voxel by a warp ballot, then union-find
// with path halving on shared indices; a tile's order is the volume's, so a tile root is its
// component's lowest flat index in the tile) and writes every voxel's tile root as its parent;
// face_union then unites only the pairs that cross a tile face, on the global parent array.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <type_traits>

#include "common.cuh"
#include "kernels.hpp"

namespace bk {

size_t label_bytes(int dtype) {
  switch (dtype) {
    case U8: case I8: return 1;
    case U16: case I16: return 2;
    case U32: case I32: return 4;
    case U64: case I64: return 8;
    default: throw std::invalid_argument("integer labels required");
  }
}

namespace {

// Root of i with path halving (every visited node is pointed at its grandparent). Parents only
// ever point to smaller indices and a shortcut only skips ancestors, so the racy writes are benign.
__device__ __forceinline__ int find_root(int *parent, int i) {
  int p = __ldcg(parent + i);
  while (p != i) {
    const int g = __ldcg(parent + p);
    if (g == p) return p;
    parent[i] = g;
    i = g;
    p = __ldcg(parent + i);
  }
  return i;
}

__device__ __forceinline__ void unite(int *parent, int a, int b) {
  a = find_root(parent, a);
  b = find_root(parent, b);
  while (a != b) {
    if (a < b) { int t = a; a = b; b = t; }  // a > b: link a under b
    const int old = atomicCAS(parent + a, a, b);
    if (old == a) return;
    a = find_root(parent, old);
    b = find_root(parent, b);
  }
}

constexpr int kTileX = 32, kTileY = 8, kTileZ = 8, kTileN = kTileX * kTileY * kTileZ, kTileThreads = 512;

// Whether the pair (p, p + (dx, dy, dz)) of equal labels is skipped: an edge pair with a face
// intermediate of the label, a corner pair with a face or edge intermediate of it. `same(a, b, c)`
// tells whether p + (a, b, c) (inside the volume) has p's label.
template <class Same>
__device__ __forceinline__ bool skipped(int dx, int dy, int dz, Same same) {
  const int nonzero = (dx != 0) + (dy != 0) + (dz != 0);
  if (nonzero == 2) return (dx && same(dx, 0, 0)) || (dy && same(0, dy, 0)) || (dz && same(0, 0, dz));
  if (nonzero == 3)
    return same(dx, 0, 0) || same(0, dy, 0) || same(0, 0, dz) || same(dx, dy, 0) || same(dx, 0, dz) || same(0, dy, dz);
  return false;
}

// Root of i in the tile's shared forest, with path halving (the same benign races as find_root).
__device__ __forceinline__ int tile_find(int *par, int i) {
  int p = par[i];
  while (p != i) {
    const int g = par[p];
    if (g == p) return p;
    par[i] = g;
    i = g;
    p = par[i];
  }
  return i;
}

__device__ __forceinline__ void tile_unite(int *par, int a, int b) {
  a = tile_find(par, a);
  b = tile_find(par, b);
  while (a != b) {
    if (a < b) { int t = a; a = b; b = t; }
    const int old = atomicCAS(par + a, a, b);
    if (old == a) return;
    a = tile_find(par, old);
    b = tile_find(par, b);
  }
}

// grid (x tiles, y tiles, z tiles from tz0); parent of every voxel of the tile = its tile root, as
// an index of the flat space the volume starts at `base` in; background: -1.
template <class L>
__global__ void __launch_bounds__(kTileThreads) tile_union(const L *__restrict__ labels, int *parent, Dims d, bool planar,
                                                           long long base, int tz0) {
  __shared__ L lab[kTileN];
  __shared__ int par[kTileN];
  const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * kTileY, z0 = (tz0 + int(blockIdx.z)) * kTileZ;
  const int ex = min(kTileX, d.sx - x0), ey = min(kTileY, d.sy - y0), ez = min(kTileZ, d.sz - z0);
  // a tile row is one warp (kTileX == 32): every voxel starts under the first voxel of its run of
  // equal labels along x, so the x-face pairs are united without a find
  static_assert(kTileX == 32 && kTileThreads % 32 == 0, "a tile row is one warp");
  for (int t = threadIdx.x; t < kTileN; t += kTileThreads) {
    const int lx = t % kTileX, ly = (t / kTileX) % kTileY, lz = t / (kTileX * kTileY);
    const bool in = lx < ex && ly < ey && lz < ez;
    const L lv = in ? labels[(x0 + lx) + (long long)d.sx * ((y0 + ly) + (long long)d.sy * (z0 + lz))] : L(0);
    lab[t] = lv;
    const L left = __shfl_up_sync(0xFFFFFFFFu, lv, 1);
    const bool joins = lx > 0 && lv != L(0) && left == lv;
    const unsigned starts = __ballot_sync(0xFFFFFFFFu, !joins);
    par[t] = t - lx + (31 - __clz(starts & (0xFFFFFFFFu >> (31 - lx))));
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kTileN; t += kTileThreads) {
    const L lv = lab[t];
    if (lv == L(0)) continue;
    const int lx = t % kTileX, ly = (t / kTileX) % kTileY, lz = t / (kTileX * kTileY);
    auto same = [&](int a, int b, int c) { return lab[t + a + kTileX * (b + kTileY * c)] == lv; };
    // Inside a region of one label: when the +y and +z neighbours (in this tile) carry the label,
    // every other forward pair has one of them as a face intermediate and is skipped, so those
    // two unions are all (in a plane, the +y one).
    if (ly + 1 < ey && same(0, 1, 0) && (planar || (lz + 1 < ez && same(0, 0, 1)))) {
      tile_unite(par, t, t + kTileX);
      if (!planar) tile_unite(par, t, t + kTileX * kTileY);
      continue;
    }
#pragma unroll
    for (int k = 0; k < 26; ++k) {
      const int dx = c_dx[k], dy = c_dy[k], dz = c_dz[k];
      if (!(dz > 0 || (dz == 0 && (dy > 0 || (dy == 0 && dx > 0))))) continue;
      if (dy == 0 && dz == 0) continue;  // the x run, linked at load
      if (planar && dz != 0) continue;
      const int nx = lx + dx, ny = ly + dy, nz = lz + dz;
      if (nx < 0 || ny < 0 || nx >= ex || ny >= ey || nz >= ez) continue;  // other tiles: face_union
      if (!same(dx, dy, dz) || skipped(dx, dy, dz, same)) continue;
      tile_unite(par, t, t + dx + kTileX * (dy + kTileY * dz));
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kTileN; t += kTileThreads) {
    const int lx = t % kTileX, ly = (t / kTileX) % kTileY, lz = t / (kTileX * kTileY);
    if (!(lx < ex && ly < ey && lz < ez)) continue;
    const int r = tile_find(par, t);
    const int rx = r % kTileX, ry = (r / kTileX) % kTileY, rz = r / (kTileX * kTileY);
    const long long g = (x0 + lx) + (long long)d.sx * ((y0 + ly) + (long long)d.sy * (z0 + lz));
    parent[base + g] = lab[t] == L(0) ? -1 : int(base + (x0 + rx) + (long long)d.sx * ((y0 + ry) + (long long)d.sy * (z0 + rz)));
  }
}

// Pairs that cross a tile face: from every voxel on a face a forward neighbour can cross (both x
// faces, both y faces — dy = -1 comes with dz = +1 — and the high z face), the forward neighbours
// in another tile; for the voxels [i0, i1) of the volume.
template <class L>
__global__ void face_union(const L *labels, int *parent, Dims d, bool planar, long long base, long long i0,
                           long long i1) {
  const long long i = i0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= i1) return;
  int x, y, z;
  unravel((int)i, d, x, y, z);
  const int lx = x % kTileX, ly = y % kTileY, lz = z % kTileZ;
  if (lx != 0 && lx != kTileX - 1 && ly != 0 && ly != kTileY - 1 && lz != kTileZ - 1) return;
  const L lv = labels[i];
  if (lv == L(0)) return;
  auto same = [&](int dx, int dy, int dz) {
    const int nx = x + dx, ny = y + dy, nz = z + dz;
    if (nx < 0 || ny < 0 || nz < 0 || nx >= d.sx || ny >= d.sy || nz >= d.sz) return false;
    return labels[i + dx + (long long)d.sx * (dy + (long long)d.sy * dz)] == lv;
  };
#pragma unroll
  for (int k = 0; k < 26; ++k) {
    const int dx = c_dx[k], dy = c_dy[k], dz = c_dz[k];
    if (!(dz > 0 || (dz == 0 && (dy > 0 || (dy == 0 && dx > 0))))) continue;
    if (planar && dz != 0) continue;
    const bool cx = lx + dx < 0 || lx + dx >= kTileX, cy = ly + dy < 0 || ly + dy >= kTileY, cz = lz + dz >= kTileZ;
    if (!(cx || cy || cz)) continue;
    if (!same(dx, dy, dz) || skipped(dx, dy, dz, same)) continue;
    // The pair one step back along an axis the pair does not cross, with both ends still inside
    // their tiles, joins the same two tile components (each end is tied to its step-back voxel
    // inside its tile) and is itself united or skipped by this rule further back; so a pair whose
    // step-back ends both carry the label adds nothing.
    long long back = 0;
    if (!cx && lx >= 1 && lx + dx >= 1) back = 1;
    else if (!cy && ly >= 1 && ly + dy >= 1) back = d.sx;
    else if (!planar && !cz && lz >= 1 && lz + dz >= 1) back = (long long)d.sx * d.sy;
    const long long q = i + nbr_offset(k, d);
    if (back && labels[i - back] == lv && labels[q - back] == lv) continue;
    unite(parent, int(base + i), int(base + q));
  }
}

__global__ void flatten(int *parent, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int p = parent[i];
  if (p < 0) return;  // background
  while (true) {
    const int q = __ldcg(parent + p);
    if (q == p) break;
    p = q;
  }
  parent[i] = p;
}

struct RootFlag {
  const int *parent;
  __device__ int operator()(long long i) const { return parent[i] == (int)i; }
};

// Each volume's first rank, and the total: bounds[v] = rank[offset_v], bounds[count] = the number
// of roots in the whole space.
__global__ void rank_bounds(const int *parent, const int *rank, const long long *offsets, int count, long long n,
                            int *bounds) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < count) bounds[v] = rank[offsets[v]];
  if (v == count) bounds[v] = rank[n - 1] + (parent[n - 1] == (int)(n - 1) ? 1 : 0);
}

// ids of one volume (local ids: rank - first + 1), and per root its local flat index and label.
template <class L>
__global__ void relabel(const L *labels, const int *parent, const int *rank, uint32_t *ids, long long *roots,
                        long long *mapping, long long n, long long base, int first) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = parent[base + i];
  if (r < 0) { ids[i] = 0; return; }
  ids[i] = uint32_t(rank[r] - first + 1);
  if (r == int(base + i)) {
    roots[rank[r]] = i;
    mapping[rank[r] + 1] = (long long)labels[i];
  }
}

template <class F>
void for_dtype(int dtype, const void *labels, F &&f) {
  switch (dtype) {
    case U8: f(static_cast<const uint8_t *>(labels)); break;
    case U16: f(static_cast<const uint16_t *>(labels)); break;
    case U32: f(static_cast<const uint32_t *>(labels)); break;
    case U64: f(static_cast<const uint64_t *>(labels)); break;
    case I8: f(static_cast<const int8_t *>(labels)); break;
    case I16: f(static_cast<const int16_t *>(labels)); break;
    case I32: f(static_cast<const int32_t *>(labels)); break;
    case I64: f(static_cast<const int64_t *>(labels)); break;
    default: throw std::invalid_argument("connected components require integer labels");
  }
}

}  // namespace

std::vector<ComponentsResult> connected_components(Context &ctx, const std::vector<CcVolume> &volumes, uint32_t *ids,
                                                   bool planar) {
  std::vector<ComponentsResult> out(volumes.size());
  long long n = 0;
  for (const auto &v : volumes) {
    if (v.offset != n) throw std::invalid_argument("component volumes must be contiguous in their flat space");
    n += v.d.n();
  }
  if (n >= (1LL << 31) - 1) throw std::invalid_argument("volumes of 2^31 voxels or more are not supported");
  for (auto &r : out) r.mapping.assign(1, 0);
  if (n <= 0) return out;
  cudaStream_t s = ctx.stream();
  Buffer<int> parent(ctx, n), rank(ctx, n);
  // union within each volume, then one flatten and one scan over all of them
  for (const auto &v : volumes) {
    if (!v.d.n()) continue;
    const Dims d{v.d.sx, v.d.sy, v.d.sz};
    const dim3 tiles((d.sx + kTileX - 1) / kTileX, (d.sy + kTileY - 1) / kTileY, (d.sz + kTileZ - 1) / kTileZ);
    if (tiles.y > 65535 || tiles.z > 65535) throw std::invalid_argument("volume too large for the tiled union");
    for_dtype(v.dtype, v.labels, [&](auto labels) {
      using L = std::remove_const_t<std::remove_pointer_t<decltype(labels)>>;
      if (!v.slabs) {
        tile_union<L><<<tiles, kTileThreads, 0, s>>>(labels, parent.data(), d, planar, v.offset, 0); ++ctx.launches;
        face_union<L><<<blocks_for(v.d.n()), 256, 0, s>>>(labels, parent.data(), d, planar, v.offset, 0, v.d.n());
        ++ctx.launches;
        return;
      }
      // labels still arriving by slabs: each slab's tiles once it is there; the cross-tile pairs
      // of a slab once the next slab (its +z neighbours) is there too
      const long long plane = (long long)d.sx * d.sy;
      int z_done = 0, z_pending = 0;  // planes united within tiles; first plane without face pairs
      for (const auto &slab : *v.slabs) {
        BK_CUDA(cudaStreamWaitEvent(s, slab.second, 0));
        const int z_end = slab.first;
        const int tz0 = z_done / kTileZ, tz1 = (z_end + kTileZ - 1) / kTileZ;
        if (tz1 > tz0) {
          tile_union<L><<<dim3(tiles.x, tiles.y, unsigned(tz1 - tz0)), kTileThreads, 0, s>>>(labels, parent.data(), d,
                                                                                             planar, v.offset, tz0);
          ++ctx.launches;
        }
        z_done = z_end;
        // planes [z_pending, z_end - 1): their +z neighbours have arrived
        const int z_ready = z_end == d.sz ? d.sz : z_end - 1;
        if (z_ready > z_pending) {
          const long long i0 = z_pending * plane, i1 = z_ready * plane;
          face_union<L><<<blocks_for(i1 - i0), 256, 0, s>>>(labels, parent.data(), d, planar, v.offset, i0, i1);
          ++ctx.launches;
          z_pending = z_ready;
        }
      }
      if (z_done != d.sz || z_pending != d.sz) throw std::logic_error("slabs do not cover the volume");
    });
  }
  flatten<<<blocks_for(n), 256, 0, s>>>(parent.data(), n); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  thrust::counting_iterator<long long> index(0);
  thrust::transform_iterator<RootFlag, thrust::counting_iterator<long long>, int> flags(index, RootFlag{parent.data()});
  size_t temp = 0;
  BK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, flags, rank.data(), n, s));
  {
    Buffer<unsigned char> scratch(ctx, temp);
    BK_CUDA(cub::DeviceScan::ExclusiveSum(scratch.data(), temp, flags, rank.data(), n, s));
  }
  std::vector<long long> offsets;
  for (const auto &v : volumes) offsets.push_back(v.offset < n ? v.offset : n - 1);
  Buffer<long long> d_offsets = to_device(ctx, offsets);
  Buffer<int> bounds(ctx, volumes.size() + 1);
  rank_bounds<<<blocks_for((long long)volumes.size() + 1), 256, 0, s>>>(parent.data(), rank.data(), d_offsets.data(),
                                                                      int(volumes.size()), n, bounds.data()); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  std::vector<int> b = bounds.download();
  for (size_t i = 0; i < volumes.size(); ++i)
    if (!volumes[i].d.n()) b[i] = i + 1 < volumes.size() ? b[i + 1] : b[volumes.size()];  // empty: no roots
  const long long total = b[volumes.size()];
  Buffer<long long> roots(ctx, total + 1), mapping(ctx, total + 1);
  for (size_t i = 0; i < volumes.size(); ++i) {
    const auto &v = volumes[i];
    if (!v.d.n()) continue;
    for_dtype(v.dtype, v.labels, [&](auto labels) {
      using L = std::remove_const_t<std::remove_pointer_t<decltype(labels)>>;
      relabel<L><<<blocks_for(v.d.n()), 256, 0, s>>>(labels, parent.data(), rank.data(), ids + v.offset, roots.data(),
                                                      mapping.data(), v.d.n(), v.offset, b[i]); ++ctx.launches;
    });
  }
  BK_CUDA(cudaGetLastError());
  const auto hr = roots.download(total), hm = mapping.download(total + 1);
  for (size_t i = 0; i < volumes.size(); ++i) {
    const long long first = b[i], count = (i + 1 < volumes.size() ? b[i + 1] : total) - first;
    out[i].count = volumes[i].d.n() ? count : 0;
    if (!out[i].count) continue;
    out[i].roots.assign(hr.begin() + first, hr.begin() + first + count);
    out[i].mapping.assign(1, 0);
    out[i].mapping.insert(out[i].mapping.end(), hm.begin() + first + 1, hm.begin() + first + 1 + count);
  }
  return out;
}

ComponentsResult connected_components(Context &ctx, const void *labels, int dtype, VolumeDims d, uint32_t *ids,
                                      bool planar) {
  label_bytes(dtype);  // rejects non-integer labels
  return connected_components(ctx, std::vector<CcVolume>{{labels, dtype, d, 0}}, ids, planar)[0];
}

}  // namespace bk
