// Connected components on sm_100a: union-find over the 13 forward neighbours of every voxel
// (the root of a component is its lowest flat index, since links always point from the larger
// root to the smaller), a read-only flatten, and ids from an exclusive scan of the root flags in
// flat order: id k belongs to the k-th root in ascending flat order, the reference's canonical
// numbering (ccl.cu:25-63 of giorgioangel/brook) without its host sort.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

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

__global__ void init_parent(int *parent, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) parent[i] = (int)i;
}

// The 13 neighbours with a positive flat offset (dz > 0, or dz == 0 and dy > 0, or dz == dy == 0
// and dx > 0). A face pair of equal labels is always united. An edge pair is skipped when one of
// its two face-adjacent intermediates has the label (the pair is then joined through it), a corner
// pair when one of its three face or three edge intermediates has it: by induction over face ->
// edge -> corner every skipped pair still ends in one component. `planar`: neighbours in the same
// z-slice only (a stack of independent 2D images).
template <class L>
__global__ void union_forward(const L *labels, int *parent, Dims d, bool planar) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n()) return;
  const L lv = labels[i];
  if (lv == 0) return;
  int x, y, z;
  unravel((int)i, d, x, y, z);
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
    if (!same(dx, dy, dz)) continue;
    const int nonzero = (dx != 0) + (dy != 0) + (dz != 0);
    if (nonzero == 2) {
      if ((dx && same(dx, 0, 0)) || (dy && same(0, dy, 0)) || (dz && same(0, 0, dz))) continue;
    } else if (nonzero == 3) {
      if (same(dx, 0, 0) || same(0, dy, 0) || same(0, 0, dz) || same(dx, dy, 0) || same(dx, 0, dz) || same(0, dy, dz))
        continue;
    }
    unite(parent, (int)i, (int)i + nbr_offset(k, d));
  }
}

__global__ void flatten(int *parent, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int p = parent[i];
  while (true) {
    const int q = __ldcg(parent + p);
    if (q == p) break;
    p = q;
  }
  parent[i] = p;
}

template <class L>
struct RootFlag {
  const L *labels;
  const int *parent;
  __device__ int operator()(long long i) const { return labels[i] != 0 && parent[i] == (int)i; }
};

// rank[n] = number of roots (the exclusive scan's total)
template <class L>
__global__ void count_roots(const L *labels, const int *parent, int *rank, long long n) {
  rank[n] = rank[n - 1] + ((labels[n - 1] != 0 && parent[n - 1] == (int)(n - 1)) ? 1 : 0);
}

template <class L>
__global__ void relabel(const L *labels, const int *parent, const int *rank, uint32_t *ids, long long *roots,
                        long long *mapping, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const L lv = labels[i];
  if (lv == 0) { ids[i] = 0; return; }
  const int r = parent[i];
  ids[i] = (uint32_t)rank[r] + 1u;
  if (r == (int)i) {
    roots[rank[i]] = i;
    mapping[rank[i] + 1] = (long long)lv;
  }
}

template <class L>
ComponentsResult run(Context &ctx, const L *labels, VolumeDims vd, uint32_t *ids, bool planar) {
  const long long n = vd.n();
  const Dims d{vd.sx, vd.sy, vd.sz};
  ComponentsResult out;
  Buffer<int> parent(ctx, n), rank(ctx, n + 1);
  cudaStream_t s = ctx.stream();
  init_parent<<<blocks_for(n), 256, 0, s>>>(parent.data(), n); ++ctx.launches;
  union_forward<L><<<blocks_for(n), 256, 0, s>>>(labels, parent.data(), d, planar); ++ctx.launches;
  flatten<<<blocks_for(n), 256, 0, s>>>(parent.data(), n); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  thrust::counting_iterator<long long> index(0);
  thrust::transform_iterator<RootFlag<L>, thrust::counting_iterator<long long>, int> flags(index, RootFlag<L>{labels, parent.data()});
  size_t temp = 0;
  BK_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, flags, rank.data(), n, s));
  Buffer<unsigned char> scratch(ctx, temp);
  BK_CUDA(cub::DeviceScan::ExclusiveSum(scratch.data(), temp, flags, rank.data(), n, s));
  count_roots<L><<<1, 1, 0, s>>>(labels, parent.data(), rank.data(), n); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  out.count = rank.download(1, n)[0];
  Buffer<long long> roots(ctx, out.count + 1), mapping(ctx, out.count + 1);
  mapping.zero();
  relabel<L><<<blocks_for(n), 256, 0, s>>>(labels, parent.data(), rank.data(), ids, roots.data(),
                                          mapping.data(), n); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  auto r = roots.download(out.count);
  auto m = mapping.download(out.count + 1);
  out.roots.assign(r.begin(), r.end());
  out.mapping.assign(m.begin(), m.end());
  return out;
}

}  // namespace

ComponentsResult connected_components(Context &ctx, const void *labels, int dtype, VolumeDims d, uint32_t *ids,
                                      bool planar) {
  if (d.n() <= 0) { ComponentsResult r; r.mapping.assign(1, 0); return r; }
  if (d.n() >= (1LL << 31) - 1) throw std::invalid_argument("volumes of 2^31 voxels or more are not supported");
  switch (dtype) {
    case U8: return run(ctx, static_cast<const uint8_t *>(labels), d, ids, planar);
    case U16: return run(ctx, static_cast<const uint16_t *>(labels), d, ids, planar);
    case U32: return run(ctx, static_cast<const uint32_t *>(labels), d, ids, planar);
    case U64: return run(ctx, static_cast<const uint64_t *>(labels), d, ids, planar);
    case I8: return run(ctx, static_cast<const int8_t *>(labels), d, ids, planar);
    case I16: return run(ctx, static_cast<const int16_t *>(labels), d, ids, planar);
    case I32: return run(ctx, static_cast<const int32_t *>(labels), d, ids, planar);
    case I64: return run(ctx, static_cast<const int64_t *>(labels), d, ids, planar);
    default: throw std::invalid_argument("connected components require integer labels");
  }
}

}  // namespace bk
