// Connected components on sm_100a: union-find over the 13 forward neighbours of every voxel
// (the root of a component is its lowest flat index, since links always point from the larger
// root to the smaller), and ids from an exclusive scan of the root flags in flat order: id k
// belongs to the k-th root in ascending flat order, the reference's canonical numbering
// (ccl.cu:25-63 of giorgioangel/brook) without its host sort.
//
// The union runs in two kernels: tile_union labels 32x8x8 tiles in shared memory (the tile's
// labels and a one-voxel halo staged once, each x run of equal labels linked to its first voxel by
// a warp ballot, then union-find with path halving on shared indices; a tile's order is the
// volume's, so a tile root is its component's lowest flat index in the tile), writes every
// voxel's tile root as its parent, and lists the pairs across tile faces that still need a union
// (from the halo, after the deduplication rules below); union_pairs then unites the listed pairs
// on the global parent array. A list that overflows its capacity falls back to face_union, which
// scans every tile-face voxel. Ids come from a scan of the root flags; relabel finds each voxel's
// root itself (no separate flatten pass).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <cstdlib>
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

// The halo of a tile: x in [x0 - 1, x0 + 32], y in [y0 - 1, y0 + 8], z in [z0, z0 + 8] (every
// forward neighbour of a tile voxel, and every intermediate of such a pair, lies inside it).
constexpr int kHaloX = kTileX + 2, kHaloY = kTileY + 2, kHaloZ = kTileZ + 1, kHaloN = kHaloX * kHaloY * kHaloZ;
constexpr int kPairStage = 512;  // cross-tile pairs a tile collects in shared memory before it writes them out

// A list of cross-tile pairs to unite: `count` entries were offered, the first `capacity` kept.
struct PairList {
  int2 *pairs;
  int *count;
  int capacity;
};

// grid (x tiles, y tiles, z tiles from tz0); parent of every voxel of the tile = its tile root, as
// an index of the flat space the volume starts at `base` in; background: -1. The cross-tile pairs
// this tile's voxels start go to `list`; pairs across the tile's +z face only where the plane
// beyond is there (z0 + 8 < z_ready).
template <class L>
__global__ void __launch_bounds__(kTileThreads, 4) tile_union(const L *__restrict__ labels, int *parent, Dims d,
                                                              bool planar, long long base, int tz0, int z_ready,
                                                              PairList list) {
  __shared__ L hal[kHaloN];
  __shared__ int par[kTileN];
  __shared__ int2 staged[kPairStage];
  __shared__ int nstaged, first;
  const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * kTileY, z0 = (tz0 + int(blockIdx.z)) * kTileZ;
  const int ex = min(kTileX, d.sx - x0), ey = min(kTileY, d.sy - y0), ez = min(kTileZ, d.sz - z0);
  const bool zface = !planar && z0 + kTileZ < d.sz && z0 + kTileZ < z_ready;
  if (threadIdx.x == 0) nstaged = 0;
  // halo load, rows of 34 along x; outside the volume (or beyond the planes this pass may read)
  // reads as background, which never equals a voxel's label
  const int hz_end = planar ? kTileZ : (zface ? kHaloZ : kTileZ);
  for (int h = threadIdx.x; h < kHaloX * kHaloY * hz_end; h += kTileThreads) {
    const int hx = h % kHaloX, hy = (h / kHaloX) % kHaloY, hz = h / (kHaloX * kHaloY);
    const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 + hz;
    const bool in = gx >= 0 && gy >= 0 && gx < d.sx && gy < d.sy && gz < d.sz;
    hal[h] = in ? labels[gx + (long long)d.sx * (gy + (long long)d.sy * gz)] : L(0);
  }
  for (int h = kHaloX * kHaloY * hz_end + threadIdx.x; h < kHaloN; h += kTileThreads) hal[h] = L(0);
  __syncthreads();
  auto at = [](int lx, int ly, int lz) { return (lx + 1) + kHaloX * ((ly + 1) + kHaloY * lz); };
  // a tile row is one warp (kTileX == 32): every voxel starts under the first voxel of its run of
  // equal labels along x, so the x-face pairs inside the tile are united without a find
  static_assert(kTileX == 32 && kTileThreads % 32 == 0, "a tile row is one warp");
  for (int t = threadIdx.x; t < kTileN; t += kTileThreads) {
    const int lx = t % kTileX, ly = (t / kTileX) % kTileY, lz = t / (kTileX * kTileY);
    const bool in = lx < ex && ly < ey && lz < ez;
    const L lv = in ? hal[at(lx, ly, lz)] : L(0);
    const bool joins = lx > 0 && lv != L(0) && hal[at(lx - 1, ly, lz)] == lv;
    const unsigned starts = __ballot_sync(0xFFFFFFFFu, !joins);
    par[t] = t - lx + (31 - __clz(starts & (0xFFFFFFFFu >> (31 - lx))));
  }
  __syncthreads();
  // Every voxel's forward pairs from its 26-bit mask of same-label neighbours. A pair is dropped
  // (1) when an intermediate voxel (a face neighbour of an edge pair, a face or edge neighbour of a
  // corner pair) carries the label: both ends are tied to it; (2) when the pair one step back along
  // x (both ends inside the tile) carries the label at both ends: those ends share x runs with this
  // pair's ends, which the load linked, and that pair is kept or dropped by the same rules further
  // back; (3) for a pair that leaves the tile and cannot step back along x, the same along y, then
  // z, since each end is tied to its step-back voxel inside its own tile. Inside a region of one
  // label only the first voxel of a tile row keeps its +y and +z pairs.
  for (int t = threadIdx.x; t < kTileN; t += kTileThreads) {
    const int lx = t % kTileX, ly = (t / kTileX) % kTileY, lz = t / (kTileX * kTileY);
    const bool in = lx < ex && ly < ey && lz < ez;
    const int h = at(lx, ly, lz);
    const L lv = in ? hal[h] : L(0);
    // only the bits the rules below read: every forward neighbour (odd k), the backward faces
    // (0, 2, 4) and the backward-y xy edges (6, 8), which corner pairs use as intermediates
    constexpr unsigned kRead = 0x2AAAAAAu | 0x155u;
    unsigned m = 0;
    if (lv != L(0)) {
#pragma unroll
      for (int k = 0; k < 26; ++k)
        if (((kRead >> k) & 1u) && lz + c_dz[k] >= 0 && hal[h + c_dx[k] + kHaloX * (c_dy[k] + kHaloY * c_dz[k])] == lv)
          m |= 1u << k;
    }
    const unsigned mprev = __shfl_up_sync(0xFFFFFFFFu, m, 1);  // the x-previous voxel's (same row)
    if (lv == L(0)) continue;
    // forward neighbours: +x (1), +y (3), +z (5), the xy edges with +y (7, 9), and every neighbour
    // with +z (11, 13, 15, 17, 19, 21, 23, 25); in-tile +x pairs are the load's run links
    unsigned cand = m & 0x2AAAAAAu & (lx == kTileX - 1 ? ~0u : ~2u);
    if (planar) cand &= 0x28Au;  // +x, +y and the xy edges with +y
    while (cand) {
      const int k = __ffs(cand) - 1;
      cand &= cand - 1;
      const int dx = c_dx[k], dy = c_dy[k], dz = c_dz[k];
      const int nz = (dx != 0) + (dy != 0) + (dz != 0);
      if (nz >= 2) {  // (1): the face intermediates, and a corner's edge intermediates
        const unsigned fx = dx ? 1u << (dx > 0 ? 1 : 0) : 0u, fy = dy ? 1u << (dy > 0 ? 3 : 2) : 0u,
                       fz = dz ? 1u << (dz > 0 ? 5 : 4) : 0u;
        unsigned inter = fx | fy | fz;
        if (nz == 3)
          inter |= (1u << (6 + ((dx > 0) << 1) + (dy > 0))) | (1u << (10 + ((dy > 0) << 1) + (dz > 0))) |
                   (1u << (14 + ((dx > 0) << 1) + (dz > 0)));
        if (m & inter) continue;
      }
      const bool cx = lx + dx < 0 || lx + dx >= kTileX, cy = ly + dy < 0 || ly + dy >= kTileY, cz = lz + dz >= kTileZ;
      const bool crossing = cx || cy || cz;
      if (cz && !zface) continue;  // the plane beyond is not here yet: face_union takes it later
      if (!cx && lx >= 1 && lx + dx >= 1) {  // (2)
        if ((m & 1u) && ((mprev >> k) & 1u)) continue;
      } else if (crossing) {  // (3)
        if (!cy && ly >= 1 && ly + dy >= 1) {
          if ((m & 4u) && hal[h + dx + kHaloX * ((dy - 1) + kHaloY * dz)] == lv) continue;
        } else if (!planar && !cz && lz >= 1 && lz + dz >= 1) {
          if ((m & 16u) && hal[h + dx + kHaloX * (dy + kHaloY * (dz - 1))] == lv) continue;
        }
      }
      if (!crossing) {
        tile_unite(par, t, t + dx + kTileX * (dy + kTileY * dz));
        continue;
      }
      const long long p = base + (x0 + lx) + (long long)d.sx * ((y0 + ly) + (long long)d.sy * (z0 + lz));
      const int2 pair = make_int2(int(p), int(p + dx + (long long)d.sx * (dy + (long long)d.sy * dz)));
      const int slot = atomicAdd(&nstaged, 1);
      if (slot < kPairStage) staged[slot] = pair;
      else if (*(volatile int *)list.count <= list.capacity) {  // more than the stage holds: to the list
        const int g = atomicAdd(list.count, 1);                    // (no more adds once it overflowed)
        if (g < list.capacity) list.pairs[g] = pair;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int n = min(nstaged, kPairStage);
    first = n && *(volatile int *)list.count <= list.capacity ? atomicAdd(list.count, n) : list.capacity;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < min(nstaged, kPairStage); i += kTileThreads)
    if (first + i < list.capacity) list.pairs[first + i] = staged[i];
  for (int t = threadIdx.x; t < kTileN; t += kTileThreads) {
    const int lx = t % kTileX, ly = (t / kTileX) % kTileY, lz = t / (kTileX * kTileY);
    if (!(lx < ex && ly < ey && lz < ez)) continue;
    const int r = tile_find(par, t);
    const int rx = r % kTileX, ry = (r / kTileX) % kTileY, rz = r / (kTileX * kTileY);
    const long long g = (x0 + lx) + (long long)d.sx * ((y0 + ly) + (long long)d.sy * (z0 + lz));
    parent[base + g] = hal[at(lx, ly, lz)] == L(0) ? -1
                                                   : int(base + (x0 + rx) + (long long)d.sx * ((y0 + ry) + (long long)d.sy * (z0 + rz)));
  }
}

// Pairs that cross a tile face: from every voxel on a face a forward neighbour can cross (both x
// faces, both y faces — dy = -1 comes with dz = +1 — and the high z face), the forward neighbours
// in another tile; for the voxels [i0, i1) of the volume.
// (The fallback of an overflowing pair list, grid-stride over [i0, i1); and, with only_z, the
// pairs across the +z faces of the tile layer whose next plane arrived after its tiles ran.)
template <class L>
__device__ void face_union_at(const L *labels, int *parent, Dims d, bool planar, long long base, long long i,
                              bool only_z) {
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
    if (!(cx || cy || cz) || (only_z && !cz)) continue;
    if (!same(dx, dy, dz) || skipped(dx, dy, dz, same)) continue;
    // the step-back rule of tile_union
    long long back = 0;
    if (!cx && lx >= 1 && lx + dx >= 1) back = 1;
    else if (!cy && ly >= 1 && ly + dy >= 1) back = d.sx;
    else if (!planar && !cz && lz >= 1 && lz + dz >= 1) back = (long long)d.sx * d.sy;
    const long long q = i + nbr_offset(k, d);
    if (back && labels[i - back] == lv && labels[q - back] == lv) continue;
    unite(parent, int(base + i), int(base + q));
  }
}

template <class L>
__global__ void face_union(const L *labels, int *parent, Dims d, bool planar, long long base, long long i0,
                           long long i1, bool only_z) {
  for (long long i = i0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < i1; i += (long long)gridDim.x * blockDim.x)
    face_union_at(labels, parent, d, planar, base, i, only_z);
}

// Unites the listed pairs; when the list overflowed, scans every tile-face voxel of the volume
// instead (face_union's rule reaches every pair the list would have held).
template <class L>
__global__ void __launch_bounds__(256, 8) union_pairs(const L *labels, int *parent, Dims d, bool planar, long long base,
                                                      long long n, PairList list) {
  const int offered = *list.count;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if (offered > list.capacity) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
      face_union_at(labels, parent, d, planar, base, i, false);
    return;
  }
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < offered; j += stride) {
    const int2 pr = list.pairs[j];
    unite(parent, pr.x, pr.y);
  }
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
  int r = parent[base + i];
  if (r < 0) { ids[i] = 0; return; }
  // a read-only walk to the root (every voxel of a tile passes through its tile root, so writing
  // shortcuts here would make thousands of threads write the same entries)
  for (int q = __ldcg(parent + r); q != r; q = __ldcg(parent + r)) r = q;
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
  // per volume: a list of cross-tile pairs (an eighth of its voxels; beyond that, face_union)
  long long forced = -1;  // test knob: a pair capacity small enough to overflow (the face_union fallback)
  if (const char *e = std::getenv("BROOK_B200_TEST_PAIR_CAPACITY")) forced = std::atoll(e);
  std::vector<long long> cap_begin(volumes.size() + 1, 0);
  for (size_t i = 0; i < volumes.size(); ++i)
    cap_begin[i + 1] = cap_begin[i] + (!volumes[i].d.n() ? 0 : forced >= 0 ? forced
                                                                  : std::max<long long>(4096, volumes[i].d.n() / 8));
  Buffer<int2> pairs(ctx, std::max<long long>(cap_begin.back(), 1));
  Buffer<int> pair_count(ctx, volumes.size());
  pair_count.zero();
  auto list_of = [&](size_t i) {
    return PairList{pairs.data() + cap_begin[i], pair_count.data() + i, int(cap_begin[i + 1] - cap_begin[i])};
  };
  // union within each volume's tiles (listing the cross-tile pairs), then the listed pairs, then
  // one scan over all volumes
  for (size_t vi = 0; vi < volumes.size(); ++vi) {
    const auto &v = volumes[vi];
    if (!v.d.n()) continue;
    const Dims d{v.d.sx, v.d.sy, v.d.sz};
    const dim3 tiles((d.sx + kTileX - 1) / kTileX, (d.sy + kTileY - 1) / kTileY, (d.sz + kTileZ - 1) / kTileZ);
    if (tiles.y > 65535 || tiles.z > 65535) throw std::invalid_argument("volume too large for the tiled union");
    const PairList list = list_of(vi);
    for_dtype(v.dtype, v.labels, [&](auto labels) {
      using L = std::remove_const_t<std::remove_pointer_t<decltype(labels)>>;
      if (!v.slabs) {
        tile_union<L><<<tiles, kTileThreads, 0, s>>>(labels, parent.data(), d, planar, v.offset, 0, d.sz, list);
        ++ctx.launches;
        return;
      }
      // labels still arriving by slabs (ends are multiples of the tiles' depth): each slab's tiles
      // once it is there, the +z face pairs of a slab's last tile layer once the next slab is too
      const long long plane = (long long)d.sx * d.sy;
      int z_done = 0;
      for (const auto &slab : *v.slabs) {
        BK_CUDA(cudaStreamWaitEvent(s, slab.second, 0));
        const int z_end = slab.first;
        const int tz0 = z_done / kTileZ, tz1 = (z_end + kTileZ - 1) / kTileZ;
        if (tz1 > tz0) {
          tile_union<L><<<dim3(tiles.x, tiles.y, unsigned(tz1 - tz0)), kTileThreads, 0, s>>>(labels, parent.data(), d,
                                                                                             planar, v.offset, tz0,
                                                                                             z_end, list);
          ++ctx.launches;
        }
        if (z_done > 0 && !planar) {  // the previous slab's last plane, now that its +z plane is here
          const long long i0 = (long long)(z_done - 1) * plane;
          face_union<L><<<blocks_for(plane), 256, 0, s>>>(labels, parent.data(), d, planar, v.offset, i0, i0 + plane,
                                                          true);
          ++ctx.launches;
        }
        z_done = z_end;
      }
      if (z_done != d.sz) throw std::logic_error("slabs do not cover the volume");
    });
  }
  for (size_t vi = 0; vi < volumes.size(); ++vi) {
    const auto &v = volumes[vi];
    if (!v.d.n()) continue;
    const Dims d{v.d.sx, v.d.sy, v.d.sz};
    for_dtype(v.dtype, v.labels, [&](auto labels) {
      using L = std::remove_const_t<std::remove_pointer_t<decltype(labels)>>;
      union_pairs<L><<<std::max(1, 8 * ctx.sm_count()), 256, 0, s>>>(labels, parent.data(), d, planar, v.offset,
                                                                     v.d.n(), list_of(vi));
      ++ctx.launches;
    });
  }
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
