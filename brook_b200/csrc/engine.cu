// Object engine kernels (see engine.hpp). A "group" — one CTA, or a cluster of 4 or 8 CTAs
// for a large object — runs one object's chain. Every frontier round has two steps separated by a
// group barrier: step A stages each frontier voxel (flag cleared, distance read, neighbour mask),
// step B spreads its 26 (voxel, neighbour) items densely over the threads, so that thousands of
// independent relaxations are in flight at once. When every CTA's share of the frontier fits its
// shared-memory staging, each CTA stages its own share there and runs only that share's items
// (an item then reads its voxel's fields without an L2 round trip); larger frontiers are staged
// in HBM and their items spread over the whole group. The group's counters live in the shared memory
// of its first CTA (distributed shared memory for a cluster, updated with 32-bit atomics only);
// 64-bit reductions (nearest rail, nearest deferred voxel, argmax) keep one copy per CTA, updated
// with CTA-local atomics and combined across the group at barriers. State other threads update
// with atomics (distances, keys, flags, staged entries) is always read through L2; state that is
// only written between floods, behind a group barrier (PDRF during a railroad flood, liveness
// during an invalidation), is read through L1, where a voxel's 26 neighbours find it again.
#include <cooperative_groups.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "common.cuh"
#include "engine.hpp"
#include "runtime.hpp"

namespace bk {
namespace {

namespace cg = cooperative_groups;

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr unsigned long long kMinFarNone = 0x7f8000007f800000ull;
constexpr unsigned long long kClaimedMark = 0xFFFFFFFFFFFFFFFEull;
// Resident engine CTAs per SM: 4 x 512 threads (full occupancy) at up to 32 registers each; the
// spills this forces cost less than the latency the extra warps hide.
constexpr int kEngineCtasPerSm = 4;

struct Shared {
  // the object (written by the group's first CTA, copied by the others)
  int obj, begin, count, status;
  int a0, sx, sy, sz;
  // group counters (used in the first CTA's copy)
  int cnt[3];  // frontier counters, a ring: current = cnt[r % 3], next = cnt[(r + 1) % 3]
  int n_far, n_keep, n_touch, flag, len;
  float T;
  unsigned long long rounds;
  // per-CTA copies, combined with Group::min_over / max_over
  unsigned long long rb, minfar, best;
  unsigned lowest, pos;
  // this CTA's copy of the object's neighbour offsets and step weights
  int off[26];
  float w[26];
  // trace: the object's root, its soma radius (< 0: none) and the loop's step (0 the soma's ball,
  // 1 the parents' field, 2 paths)
  double soma_radius;
  int root, step;
  float rscale, rconst;  // invalidation: reach = rscale * DBF[source] + rconst
  int skipped;           // manual targets from which no rail was reachable (empty paths)
};

__device__ __forceinline__ float inf() { return __uint_as_float(BK_INF_BITS); }

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void unravel3(int i, int sx, int sy, int &x, int &y, int &z) {
  const int sxy = sx * sy;
  z = i / sxy;
  const int r = i - z * sxy;
  y = r / sx;
  x = r - y * sx;
}

__device__ __forceinline__ unsigned long long pack3(int x, int y, int z) {
  return (unsigned long long)x | ((unsigned long long)y << 21) | ((unsigned long long)z << 42);
}
__device__ __forceinline__ void unpack3(unsigned long long p, int &x, int &y, int &z) {
  x = int(p & 0x1FFFFF);
  y = int((p >> 21) & 0x1FFFFF);
  z = int(p >> 42);
}

// A group of C CTAs working on one object. For C == 1 it is the CTA.
template <int C>
struct Group {
  __device__ static int rank() {
    if constexpr (C == 1) return 0;
    else return int(cg::this_cluster().block_rank());
  }
  __device__ static void sync() {
    if constexpr (C == 1) __syncthreads();
    else cg::this_cluster().sync();
  }
  __device__ static Shared *leader(Shared *own) {
    if constexpr (C == 1) return own;
    else return cg::this_cluster().map_shared_rank(own, 0);
  }
  __device__ static int tid() { return rank() * int(blockDim.x) + int(threadIdx.x); }
  // Least / greatest of the group's copies of a per-CTA field (plain loads; call between barriers).
  __device__ static unsigned long long min_over(unsigned long long *own) {
    if constexpr (C == 1) return *(volatile unsigned long long *)own;
    else {
      unsigned long long r = ~0ull;
      for (int q = 0; q < C; ++q) {
        const unsigned long long v = *(volatile unsigned long long *)cg::this_cluster().map_shared_rank(own, q);
        r = v < r ? v : r;
      }
      return r;
    }
  }
  __device__ static unsigned min_over(unsigned *own) {
    if constexpr (C == 1) return *(volatile unsigned *)own;
    else {
      unsigned r = ~0u;
      for (int q = 0; q < C; ++q) {
        const unsigned v = *(volatile unsigned *)cg::this_cluster().map_shared_rank(own, q);
        r = v < r ? v : r;
      }
      return r;
    }
  }
  __device__ static unsigned long long max_over(unsigned long long *own) {
    if constexpr (C == 1) return *(volatile unsigned long long *)own;
    else {
      unsigned long long r = 0;
      for (int q = 0; q < C; ++q) {
        const unsigned long long v = *(volatile unsigned long long *)cg::this_cluster().map_shared_rank(own, q);
        r = v > r ? v : r;
      }
      return r;
    }
  }
  __device__ static int threads() { return C * int(blockDim.x); }
  __device__ static bool first() { return rank() == 0 && threadIdx.x == 0; }
};

template <class T>
__device__ __forceinline__ T vload(const T *p) { return *(const volatile T *)p; }

// A loop bound, lowered to the test cap when one is set.
__device__ __forceinline__ long long capped(const EngineArgs &a, long long bound) {
  return a.round_limit > 0 && a.round_limit < bound ? a.round_limit : bound;
}

// Per-CTA staging of a round's frontier in shared memory. When every CTA's share of the frontier
// fits, a CTA stages its own share (step A) and spreads only that share's (voxel, neighbour) items
// over its threads (step B): the items then read their voxel's staged fields from shared memory
// instead of L2, which takes one to four dependent L2 round trips out of every item's chain.
// Larger frontiers go through the global staging arrays, items spread over the whole group.
constexpr int kStageBytes = 18432;
constexpr int kFloodStage = kStageBytes / 12;  // distance|mask (8) + voxel (4)
constexpr int kInvalStage = kStageBytes / 36;  // key (8) + both positions (16) + voxel, mask, reach (12)
constexpr int kBandStage = kStageBytes / 24;   // best offer (8) + position (8) + voxel, mask (8)

__device__ __forceinline__ unsigned char *stage_bytes() {
  __shared__ __align__(16) unsigned char buf[kStageBytes];
  return buf;
}

// This CTA's share [lo, hi) of n entries, when the largest share fits `cap` (the same answer in
// every CTA of the group, which all read the same n).
template <int C>
__device__ __forceinline__ bool own_share(int n, int cap, int &lo, int &hi) {
  if ((n + C - 1) / C > cap) return false;
  const int r = Group<C>::rank();
  lo = int((long long)n * r / C);
  hi = int((long long)n * (r + 1) / C);
  return true;
}

// Pulls the next object for this group; false when its queue is empty. The group's first CTA
// pops and publishes; every CTA copies the object into its own shared memory.
template <int C>
__device__ bool next_object(const EngineArgs &a, Shared &sh, Shared *L, bool big) {
  using G = Group<C>;
  if (G::first()) {
    const int j = atomicAdd(a.queue + (big ? 0 : 1), 1);
    const int limit = big ? a.nbig : a.nobj - a.nbig;
    L->obj = j < limit ? a.schedule[big ? j : a.nbig + j] : -1;
    if (L->obj >= 0) {
      const int o = L->obj;
      L->begin = a.obj_begin[o];
      L->count = a.obj_count[o];
      L->status = a.status[o];  // kOk unless an earlier pass gave up on the object
      const int r = a.obj_arena[o];
      L->a0 = a.arena_offset[r];
      L->sx = a.arena_dims[3 * r];
      L->sy = a.arena_dims[3 * r + 1];
      L->sz = a.arena_dims[3 * r + 2];
    }
  }
  G::sync();
  if (threadIdx.x == 0) {
    sh.obj = vload(&L->obj);
    if (sh.obj >= 0) {
      sh.begin = vload(&L->begin); sh.count = vload(&L->count);
      sh.a0 = vload(&L->a0); sh.sx = vload(&L->sx); sh.sy = vload(&L->sy); sh.sz = vload(&L->sz);
    }
  }
  __syncthreads();
  if (sh.obj >= 0 && threadIdx.x < 26) {
    const int k = threadIdx.x;
    sh.off[k] = c_dx[k] + sh.sx * (c_dy[k] + sh.sy * c_dz[k]);
    sh.w[k] = a.w[k];
  }
  // every CTA has its copy before the first CTA moves on (or exits, ending its shared memory)
  G::sync();
  return sh.obj >= 0;
}

// ---------------------------------------------------------------------------------------------
// Geometric flood from `source` over the object's voxels into `d` (+inf at rest on them):
// Bellman-Ford rounds, fl(d[u] + w[k]). The fixed point is the least float32 path sum, which any
// schedule reaches. Returns false when the round bound is hit.
// The free-space seed of a soma's DAF (sssp_kernels.cuh:14-35): the 26-connected distance from
// the root through empty space, for voxels within `radius` (float32 physical distance) of it;
// -1 beyond. One rounding per operation, in the reference's order.
__device__ float freespace_seed(const EngineArgs &a, int x, int y, int z, int rx, int ry, int rz, float radius) {
  const float wx = a.wx, wy = a.wy, wz = a.wz;
  const float rdx = __fmul_rn(wx, float(x - rx)), rdy = __fmul_rn(wy, float(y - ry)), rdz = __fmul_rn(wz, float(z - rz));
  const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(rdx, rdx), __fmul_rn(rdy, rdy)), __fmul_rn(rdz, rdz));
  if (r2 > __fmul_rn(radius, radius)) return -1.0f;
  const float dx = fabsf(float(x - rx)), dy = fabsf(float(y - ry)), dz = fabsf(float(z - rz));
  const float dxyz = fminf(fminf(dx, dy), dz);
  const float dxy = fminf(dx, dy), dyz = fminf(dy, dz), dxz = fminf(dx, dz);
  const float wxx = __fmul_rn(wx, wx), wyy = __fmul_rn(wy, wy), wzz = __fmul_rn(wz, wz);
  float v = __fmul_rn(dxyz, sqrtf(__fadd_rn(__fadd_rn(wxx, wyy), wzz)));
  v = __fadd_rn(v, __fmul_rn(wx, __fsub_rn(dx, dxyz)));
  v = __fadd_rn(v, __fmul_rn(wy, __fsub_rn(dy, dxyz)));
  v = __fadd_rn(v, __fmul_rn(wz, __fsub_rn(dz, dxyz)));
  v = __fadd_rn(v, __fmul_rn(__fsub_rn(dxy, dxyz), __fsub_rn(__fsub_rn(sqrtf(__fadd_rn(wxx, wyy)), wx), wy)));
  v = __fadd_rn(v, __fmul_rn(__fsub_rn(dxz, dxyz), __fsub_rn(__fsub_rn(sqrtf(__fadd_rn(wxx, wzz)), wx), wz)));
  v = __fadd_rn(v, __fmul_rn(__fsub_rn(dyz, dxyz), __fsub_rn(__fsub_rn(sqrtf(__fadd_rn(wyy, wzz)), wy), wz)));
  return v;
}

// seed_radius > 0 (a soma's DAF): every object voxel within it of `source` starts at its
// free-space seed, and the rounds relax from all of them.
template <int C>
__device__ bool flood_geometric(const EngineArgs &a, Shared &sh, Shared *L, float *d, int source, int *A, int *B,
                                unsigned long long *wide, float seed_radius = 0.0f) {
  using G = Group<C>;
  if (G::first()) { L->cnt[0] = 0; L->cnt[1] = 0; L->cnt[2] = 0; }
  G::sync();
  if (seed_radius > 0.0f) {
    int rx, ry, rz;
    unravel3(source - sh.a0, sh.sx, sh.sy, rx, ry, rz);
    for (int i = G::tid(); i < sh.count; i += G::threads()) {
      const int v = a.vox[sh.begin + i];
      int x, y, z;
      unravel3(v - sh.a0, sh.sx, sh.sy, x, y, z);
      const float s = freespace_seed(a, x, y, z, rx, ry, rz, seed_radius);
      if (s < 0.0f) continue;
      d[v] = s;
      atomicOr(a.flags + v, kNearQueued);
      A[atomicAdd(&L->cnt[0], 1)] = v;
    }
  } else if (G::first()) {
    d[source] = 0.0f;
    atomicOr(a.flags + source, kNearQueued);
    A[0] = source;
    L->cnt[0] = 1;
  }
  G::sync();
  const long long bound = capped(a, 8LL * sh.count + 256);
  for (int r = 0;; ++r) {
    int *cur = (r & 1) ? B : A, *nxt = (r & 1) ? A : B;
    const int nc = vload(&L->cnt[r % 3]);
    if (nc == 0) break;
    if (r >= bound) return false;
    if (G::first()) L->cnt[(r + 2) % 3] = 0;
    int *next_count = &L->cnt[(r + 1) % 3];
    auto relax = [&](unsigned long long e, int u, int k) {
      if (!((unsigned(e) >> k) & 1u)) return;
      const int v = u + sh.off[k];
      const float cand = __fadd_rn(__uint_as_float(unsigned(e >> 32)), sh.w[k]);
      const float old = atomic_min_pos(d + v, cand);
      if (old > cand && !(atomicOr(a.flags + v, kNearQueued) & kNearQueued)) nxt[atomicAdd(next_count, 1)] = v;
    };
    // step A runs between barriers, with no relaxation in flight: the flag clear (a reduction,
    // nothing to wait for) and the distance read need no order between them
    int lo, hi;
    if (own_share<C>(nc, kFloodStage, lo, hi)) {
      unsigned long long *se = reinterpret_cast<unsigned long long *>(stage_bytes());
      int *su = reinterpret_cast<int *>(se + kFloodStage);
      for (int i = lo + int(threadIdx.x); i < hi; i += blockDim.x) {
        const int u = __ldcg(cur + i);
        atomicAnd(a.flags + u, ~kNearQueued);
        const float du = __ldcg(d + u);
        su[i - lo] = u;
        se[i - lo] = (static_cast<unsigned long long>(__float_as_uint(du)) << 32) | a.mask[u];
      }
      G::sync();
      for (int j = threadIdx.x; j < (hi - lo) * 26; j += blockDim.x) {
        const int q = j / 26;
        relax(se[q], su[q], j - 26 * q);
      }
    } else {
      for (int i = G::tid(); i < nc; i += G::threads()) {
        const int u = __ldcg(cur + i);
        atomicAnd(a.flags + u, ~kNearQueued);
        const float du = __ldcg(d + u);
        wide[i] = (static_cast<unsigned long long>(__float_as_uint(du)) << 32) | a.mask[u];
      }
      G::sync();
      for (long long j = G::tid(); j < (long long)nc * 32; j += G::threads()) {
        const int k = int(j & 31);
        if (k >= 26) continue;
        const int i = int(j >> 5);
        relax(__ldcg(wide + i), __ldcg(cur + i), k);
      }
    }
    G::sync();
  }
  return true;
}

// Largest finite value of `f` over the object's voxels, ties -> lowest flat index: the packed key
// (value bits << 32 | ~flat), 0 when nothing is finite.
template <int C>
__device__ unsigned long long object_argmax(const EngineArgs &a, Shared &sh, Shared *L, const float *f) {
  using G = Group<C>;
  if (threadIdx.x == 0) sh.best = 0;
  G::sync();
  unsigned long long best = 0;
  for (int i = G::tid(); i < sh.count; i += G::threads()) {
    const int v = a.vox[sh.begin + i];
    const float x = __ldcg(f + v);
    if (x < inf()) {
      const unsigned long long k = (static_cast<unsigned long long>(__float_as_uint(x)) << 32) | (0xFFFFFFFFu - unsigned(v));
      best = k > best ? k : best;
    }
  }
  const unsigned hi = __reduce_max_sync(kFull, unsigned(best >> 32));
  const unsigned lo = __reduce_max_sync(kFull, unsigned(best >> 32) == hi ? unsigned(best) : 0u);
  if ((threadIdx.x & 31) == 0) atomicMax(&sh.best, (static_cast<unsigned long long>(hi) << 32) | lo);
  G::sync();
  const unsigned long long r = G::max_over(&sh.best);
  G::sync();
  return r;
}

template <int C>
__device__ void prepare_loop(const EngineArgs &a, bool big) {
  using G = Group<C>;
  __shared__ Shared sh;
  Shared *L = G::leader(&sh);
  while (next_object<C>(a, sh, L, big)) {
    const int o = sh.obj;
    int *A = a.lists + sh.begin, *B = a.lists + a.F + sh.begin;
    unsigned long long *wide = a.wide + sh.begin;
    int root = a.border_root[o];
    bool ok = true;
    if (root < 0) {
      // the farthest voxel (geometric distance) from the object's first voxel
      ok = flood_geometric<C>(a, sh, L, a.daf, a.vox[sh.begin], A, B, wide);
      if (ok) {
        const unsigned long long k = object_argmax<C>(a, sh, L, a.daf);
        root = int(0xFFFFFFFFu - unsigned(k));
        for (int i = G::tid(); i < sh.count; i += G::threads()) a.daf[a.vox[sh.begin + i]] = inf();
        G::sync();
      }
    }
    if (ok) ok = flood_geometric<C>(a, sh, L, a.daf, root, A, B, wide, a.free_radius[o]);
    if (!ok) {
      if (G::first()) a.status[o] = kBudget;
      G::sync();
      continue;
    }
    const unsigned long long k = object_argmax<C>(a, sh, L, a.daf);
    const float farthest = __uint_as_float(unsigned(k >> 32));
    const int target = int(0xFFFFFFFFu - unsigned(k));
    // PDRF of the object's voxels (the reference's pdrf_lab, batched_regular.inc:93-108):
    // (1 - dbf * M)^(2^squarings) * scale + daf * inv, one rounding per operation.
    const float M = a.M[o];
    const bool with_daf = farthest != 0.0f;
    const float inv = with_daf ? __double2float_rn(__ddiv_rn(1.0, (double)farthest)) : 0.0f;
    for (int i = G::tid(); i < sh.count; i += G::threads()) {
      const int v = a.vox[sh.begin + i];
      a.pdrf[v] = pdrf_value(a.dbf[v], with_daf ? __ldcg(a.daf + v) : 0.0f, M, inv, a.pdrf_scale, a.squarings,
                             a.exponent);
    }
    G::sync();
    if (G::first()) {
      if (a.fix_branching) a.pdrf[root] = 0.0f;  // the root is the first rail
      a.root[o] = root;
      a.target[o] = target;
      a.max_daf[o] = farthest;
    }
    G::sync();
  }
}

// Every CTA belongs to a cluster. The clusters first take the large objects, one each, then every
// CTA takes small objects on its own: large objects start first (they set the kernel's length),
// and no CTA idles while any object is left.
template <int C>
__global__ void __launch_bounds__(kEngineThreads, kEngineCtasPerSm) prepare_kernel(EngineArgs a) {
  prepare_loop<C>(a, true);
  prepare_loop<1>(a, false);
}

// ---------------------------------------------------------------------------------------------
// Railroad flood from target t over the object's voxels: entering v costs pdrf[v] (vw_step), rails
// (pdrf == 0) absorb. Near-far bands: the near band [.., T] is relaxed to convergence, bounded by
// the best rail found so far; the next band starts at the nearest deferred voxel. Returns the
// nearest rail as (distance bits << 32 | flat), BK_UNCLAIMED when no rail is reachable, and sets
// L->status on a bound. The result is schedule-independent: every voxel at distance <= D (the
// nearest rail's) is exact when the flood stops.
template <int C>
__device__ unsigned long long railroad(const EngineArgs &a, Shared &sh, Shared *L, int t, int *A, int *B, int *FA,
                                       int *FB, int *touched, unsigned long long *wide) {
  using G = Group<C>;
  // without fix_branching there are no rails: a full SSSP from t (the parents' field)
  if (threadIdx.x == 0) {
    sh.rb = BK_UNCLAIMED;
    sh.minfar = kMinFarNone;
  }
  if (G::first()) {
    L->n_touch = 1;
    touched[0] = t;
    L->cnt[0] = 0; L->cnt[1] = 0; L->cnt[2] = 0;
    L->n_far = 0; L->n_keep = 0;
    a.dist[t] = 0.0f;
    const float ft = __ldcg(a.pdrf + t);
    if (a.fix_branching && ft == 0.0f) sh.rb = static_cast<unsigned long long>(unsigned(t));
    else {
      A[0] = t;
      L->cnt[0] = 1;
      atomicOr(a.flags + t, kNearQueued);
      L->T = fmaxf(__fmul_rn(a.rail_band, ft), 1e-30f);
    }
  }
  G::sync();
  {
    const unsigned long long rb = G::min_over(&sh.rb);
    if (rb != BK_UNCLAIMED) {
      G::sync();
      return rb;
    }
  }
  int *far = FA, *keep = FB;
  const long long bound = capped(a, 16LL * sh.count + 256);
  long long work = 0;
  int r = 0;
  for (;;) {
    for (;; ++r) {
      int *cur = (r & 1) ? B : A, *nxt = (r & 1) ? A : B;
      const int nc = vload(&L->cnt[r % 3]);
      if (nc == 0) break;
      if (++work > bound) {
        if (G::first()) L->status = kBudget;
        G::sync();
        return BK_UNCLAIMED;
      }
      if (G::first()) { L->cnt[(r + 2) % 3] = 0; L->rounds += 1; }
      const float T = vload(&L->T);
      int *next_count = &L->cnt[(r + 1) % 3];
      // step A: no relaxation is in flight between the barriers
      auto stage = [&](int u) {
        atomicAnd(a.flags + u, ~kNearQueued);
        const float fu = a.pdrf[u];
        const float du = __ldcg(a.dist + u);
        const unsigned long long rb = vload(&sh.rb);
        const float Tb = rb != BK_UNCLAIMED ? fminf(T, __uint_as_float(unsigned(rb >> 32))) : T;
        const bool expand = (fu != 0.0f || !a.fix_branching) && du <= Tb;
        return expand ? (static_cast<unsigned long long>(__float_as_uint(du)) << 32) | a.mask[u] : 0ull;
      };
      // step B, after the improvement of v to cand (from old)
      auto improved = [&](int v, float cand, float fv, float old) {
        {
          if (old == inf()) touched[atomicAdd(&L->n_touch, 1)] = v;
          if (a.fix_branching && fv == 0.0f)
            atomicMin(&sh.rb, (static_cast<unsigned long long>(__float_as_uint(cand)) << 32) | unsigned(v));
          const unsigned long long rb = vload(&sh.rb);
          const float Tb = rb != BK_UNCLAIMED ? fminf(T, __uint_as_float(unsigned(rb >> 32))) : T;
          if (cand <= Tb) {
            if (!(atomicOr(a.flags + v, kNearQueued) & kNearQueued)) nxt[atomicAdd(next_count, 1)] = v;
          } else {
            atomicMin(&sh.minfar, (static_cast<unsigned long long>(__float_as_uint(cand)) << 32) | __float_as_uint(fv));
            if (!(atomicOr(a.flags + v, kFarQueued) & kFarQueued)) far[atomicAdd(&L->n_far, 1)] = v;
          }
        }
      };
      // step B: one (voxel, neighbour) item
      auto relax = [&](unsigned long long e, int u, int k) {
        if (!((unsigned(e) >> k) & 1u)) return;
        const int v = u + sh.off[k];
        const float fv = a.pdrf[v];
        const float cand = vw_step(__uint_as_float(unsigned(e >> 32)), fv);
        const float old = atomic_min_pos(a.dist + v, cand);
        if (old > cand) improved(v, cand, fv, old);
      };
      int lo, hi;
      if (own_share<C>(nc, kFloodStage, lo, hi)) {
        unsigned long long *se = reinterpret_cast<unsigned long long *>(stage_bytes());
        int *su = reinterpret_cast<int *>(se + kFloodStage);
        for (int i = lo + int(threadIdx.x); i < hi; i += blockDim.x) {
          const int u = __ldcg(cur + i);
          su[i - lo] = u;
          se[i - lo] = stage(u);
        }
        G::sync();
        for (int j = threadIdx.x; j < (hi - lo) * 26; j += blockDim.x) {
          const int q = j / 26;
          relax(se[q], su[q], j - 26 * q);
        }
      } else {
        for (int i = G::tid(); i < nc; i += G::threads()) wide[i] = stage(__ldcg(cur + i));
        G::sync();
        for (long long j = G::tid(); j < (long long)nc * 32; j += G::threads()) {
          const int k = int(j & 31);
          if (k >= 26) continue;
          const int i = int(j >> 5);
          relax(__ldcg(wide + i), __ldcg(cur + i), k);
        }
      }
      G::sync();
    }
    // band end: the nearest rail is final once it lies inside the band
    if (G::first()) {
      L->flag = 0;
      const unsigned long long rb = G::min_over(&sh.rb), minfar = G::min_over(&sh.minfar);
      sh.rb = rb;
      if (rb != BK_UNCLAIMED && __uint_as_float(unsigned(rb >> 32)) <= L->T) L->flag = 1;
      else if (minfar == kMinFarNone) L->flag = 2;
      else {
        const float d = __uint_as_float(unsigned(minfar >> 32)), f = __uint_as_float(unsigned(minfar));
        float w = __fmul_rn(a.rail_band, f);
        const float lo = __fmul_rn(5e-4f, d);
        if (!(w > lo)) w = lo;
        L->T = __fadd_rn(d, w);
      }
      L->n_keep = 0;
    }
    G::sync();
    // every CTA takes the combined rail and starts a fresh nearest-deferred minimum
    if (threadIdx.x == 0) {
      if (G::rank() != 0) sh.rb = vload(&L->rb);
      sh.minfar = kMinFarNone;
    }
    __syncthreads();
    const int flag = vload(&L->flag);
    if (flag) {
      const unsigned long long rb = vload(&sh.rb);
      G::sync();
      return flag == 1 ? rb : BK_UNCLAIMED;
    }
    // promote deferred voxels inside the new band into the current near list
    int *cur = (r & 1) ? B : A;
    const int nf = vload(&L->n_far);
    const unsigned long long rb = vload(&sh.rb);
    const float T = vload(&L->T);
    const float Tp = rb != BK_UNCLAIMED ? fminf(T, __uint_as_float(unsigned(rb >> 32))) : T;
    int *cur_count = &L->cnt[r % 3];
    for (int i = G::tid(); i < nf; i += G::threads()) {
      const int w = __ldcg(far + i);
      const float dw = __ldcg(a.dist + w);
      if (dw <= Tp) {
        atomicAnd(a.flags + w, ~kFarQueued);
        if (!(atomicOr(a.flags + w, kNearQueued) & kNearQueued)) cur[atomicAdd(cur_count, 1)] = w;
      } else {
        atomicMin(&sh.minfar, (static_cast<unsigned long long>(__float_as_uint(dw)) << 32) | __float_as_uint(a.pdrf[w]));
        keep[atomicAdd(&L->n_keep, 1)] = w;
      }
    }
    G::sync();
    if (G::first()) L->n_far = L->n_keep;
    int *tmp = far; far = keep; keep = tmp;
    G::sync();
  }
}

// One warp walks from the nearest rail back to the target: the step goes to the neighbour of least
// distance (non-rail, lowest neighbour index among ties); at the first step the rail end is
// re-picked as the last road voxel's first rail in dijkstra3d order (lockstep_regular.inc:61-155).
// Writes the path target-first to out and returns its length (-1: no room).
__device__ int backtrace(const EngineArgs &a, const Shared &sh, unsigned long long rb, int t, int *out, long long room) {
  const int lane = threadIdx.x & 31;
  int cur = int(unsigned(rb));
  int len = 0;
  const long long bound = 2LL * sh.count + 2;
  for (long long step = 0; step < bound; ++step) {
    int kb = -1;
    if (cur != t) {
      const uint32_t m = a.mask[cur];
      unsigned db = BK_INF_BITS;
      if (lane < 26 && ((m >> lane) & 1u)) {
        const int u = cur + sh.off[lane];
        if (a.pdrf[u] != 0.0f) db = __float_as_uint(__ldcg(a.dist + u));
      }
      const unsigned mb = __reduce_min_sync(kFull, db);
      if (mb < BK_INF_BITS) kb = int(__reduce_min_sync(kFull, db == mb ? unsigned(lane) : 64u));
    }
    if (step == 0 && kb >= 0) {
      const int u = cur + sh.off[kb];
      const uint32_t mu = a.mask[u];
      unsigned key = 64;
      if (lane < 26 && ((mu >> lane) & 1u) && a.pdrf[u + sh.off[lane]] == 0.0f) key = unsigned(c_d3rank[lane]);
      const unsigned r = __reduce_min_sync(kFull, key);
      if (r < 26) {
        const int ks = c_d3inv[r];
        cur = u + sh.off[ks];
        kb = c_opp[ks];
      }
    }
    if (len >= room) return -1;
    if (lane == 0) out[len] = cur;
    ++len;
    if (kb < 0) break;
    cur += sh.off[kb];
  }
  __syncwarp();
  for (int i = lane; i < len / 2; i += 32) {
    const int x = out[i];
    out[i] = out[len - 1 - i];
    out[len - 1 - i] = x;
  }
  __syncwarp();
  return len;
}

// Without fix_branching: one warp walks from target t to the root through the parents' field (the
// object's SSSP distances from the root): each step goes to the neighbour of least distance,
// lowest neighbour index among ties (vw_assign_parents, sssp_kernels.cuh:89-110). Writes the path
// target-first to out and returns its length (-1: no room). The walk stops at the first voxel of
// an earlier path (kOnPath): the parents' field is a tree, so from there it would repeat that
// path's tail, whose vertices and edges the skeleton already holds and whose voxels are already
// dead (no invalidation source); the stored paths then total at most the object's voxels plus
// one per path.
__device__ int parent_walk(const EngineArgs &a, const Shared &sh, int t, int root, int *out, long long room) {
  const int lane = threadIdx.x & 31;
  int cur = t;
  int len = 0;
  const long long bound = 2LL * sh.count + 2;
  for (long long step = 0; step < bound; ++step) {
    if (len >= room) return -1;
    if (lane == 0) out[len] = cur;
    ++len;
    if (cur == root || (__ldcg(a.flags + cur) & kOnPath) || !(__ldcg(a.dist + cur) < inf())) break;
    const uint32_t m = a.mask[cur];
    unsigned db = BK_INF_BITS;
    if (lane < 26 && ((m >> lane) & 1u)) db = __float_as_uint(__ldcg(a.dist + cur + sh.off[lane]));
    const unsigned mb = __reduce_min_sync(kFull, db);
    if (!(mb < BK_INF_BITS)) break;
    cur += sh.off[__reduce_min_sync(kFull, db == mb ? unsigned(lane) : 64u)];
  }
  __syncwarp();
  return len;
}

// Soma trimming of a stored path (trace.cu:222-236), one warp, in place. A vertex is far when its
// float64 physical distance from the root exceeds the soma radius. With fix_branching (a
// target-first railroad path) the first vertex stays, then every far vertex, then the root when
// the rail end is not far. Without it (a target-first walk that stopped at w, the root or a vertex
// of an earlier trimmed path) the far vertices before w stay, then w: the reference's root-first
// path [root, far vertices] joins the earlier paths exactly there (its far vertices beyond w are
// those paths' own). Returns the new length (-1: no room).
__device__ int soma_trim(const EngineArgs &a, const Shared &sh, int *path, int len, int root, double radius, bool rails,
                         long long room) {
  const int lane = threadIdx.x & 31;
  int rx, ry, rz;
  unravel3(root - sh.a0, sh.sx, sh.sy, rx, ry, rz);
  auto far = [&](int v) {
    int x, y, z;
    unravel3(v - sh.a0, sh.sx, sh.sy, x, y, z);
    const double dx = __dmul_rn(double(a.wx), double(x - rx)), dy = __dmul_rn(double(a.wy), double(y - ry)),
                 dz = __dmul_rn(double(a.wz), double(z - rz));
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz))) > radius;
  };
  const int last = path[len - 1];
  const bool last_far = far(last);
  // the kept range: [1, len) with the first vertex kept as it is (rails), or [0, len - 1) with the
  // stop vertex appended (no rails)
  const int begin = rails ? 1 : 0, end = rails ? len : len - 1;
  int k = rails ? 1 : 0;
  for (int base = begin; base < end; base += 32) {
    const int i = base + lane;
    const int v = i < end ? path[i] : 0;
    const bool keep = i < end && far(v);
    const unsigned ballot = __ballot_sync(kFull, keep);
    __syncwarp();
    if (keep) path[k + __popc(ballot & ((1u << lane) - 1u))] = v;
    k += __popc(ballot);
    __syncwarp();
  }
  if (rails && !last_far) {
    if (k >= room) return -1;
    if (lane == 0) path[k] = root;
    ++k;
  } else if (!rails) {
    if (lane == 0) path[k] = last;
    ++k;
  }
  __syncwarp();
  return k;
}

__device__ __forceinline__ float distance_to(const EngineArgs &a, int x, int y, int z, int qx, int qy, int qz) {
  const float dx = __fmul_rn(a.wx, float(x - qx)), dy = __fmul_rn(a.wy, float(y - qy)), dz = __fmul_rn(a.wz, float(z - qz));
  return sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}
__device__ __forceinline__ float reach(const EngineArgs &a, int s, float scale, float constant) {
  return __fadd_rn(__fmul_rn(scale, a.dbf[s]), constant);
}
__device__ __forceinline__ int band_of(unsigned mbits, float delta, int kmin) {
  const float m = __uint_as_float(mbits);
  int k = int(__fdiv_rn(m, delta));
  while (__fmul_rn(float(k + 1), delta) <= m) ++k;
  while (k > 0 && __fmul_rn(float(k), delta) > m) --k;
  return k < kmin ? kmin : k;
}

// Claim-order invalidation of one path (invalidation_kernels.cuh:105-297; lockstep_coop.inc:530-845):
// alive path vertices become sources (bottleneck M = 0); a claimed voxel u holding (M, s) offers
// an alive neighbour v the source s when |aniso (v - s)| < scale DBF[s] + const, with
// M' = max(M, |v - s|). Inside the band [k delta, (k+1) delta) offers claim at once, keeping the
// least (M bits, source); rounds are synchronous (offers come from the keys of the round
// boundary). Offers beyond the band wait; at the boundary each waiting voxel takes the best offer
// of its claimed neighbours, the smallest names the next band, those inside it are claimed.
// Claimed voxels die. Returns false when a loop bound is hit.
template <int C>
__device__ bool invalidate(const EngineArgs &a, Shared &sh, Shared *L, const int *path, int npath, int *A, int *B,
                           int *FA, int *FB, int *touched, unsigned long long *wide, unsigned long long *side_u,
                           unsigned long long *side_s) {
  using G = Group<C>;
  if (G::first()) { L->cnt[0] = 0; L->cnt[1] = 0; L->cnt[2] = 0; L->n_far = 0; L->n_keep = 0; L->n_touch = 0; }
  G::sync();
  for (int i = G::tid(); i < npath; i += G::threads()) {
    const int p = __ldcg(path + i);
    if (!__ldcg(a.alive + p)) continue;
    const unsigned long long old = atomicMin(a.key + p, static_cast<unsigned long long>(unsigned(p)));
    if (old == BK_UNCLAIMED) {
      atomicOr(a.flags + p, kFront);
      A[atomicAdd(&L->cnt[0], 1)] = p;
      touched[atomicAdd(&L->n_touch, 1)] = p;
    }
  }
  G::sync();
  int *far = FA, *keep = FB;
  const long long bound = capped(a, 64LL * sh.count + 1024);
  long long work = 0;
  int band = 0, r = 0;
  for (;;) {
    unsigned hi = __float_as_uint(__fmul_rn(float(band + 1), a.delta));
    for (;; ++r) {
      int *cur = (r & 1) ? B : A, *nxt = (r & 1) ? A : B;
      const int nc = vload(&L->cnt[r % 3]);
      if (nc == 0) break;
      if (++work > bound) return false;
      if (G::first()) { L->cnt[(r + 2) % 3] = 0; L->rounds += 1ull << 32; }
      int *next_count = &L->cnt[(r + 1) % 3];
      // step B: the offer of claimed u (key ku, positions (ux, uy, uz) and its source's, the
      // source's reach) to its k-th neighbour; distance and reach checks come before the read of
      // the neighbour's liveness (all three only filter)
      auto offer = [&](int u, unsigned long long ku, int k, int ux, int uy, int uz, int qx, int qy, int qz, float rs) {
        const float d = distance_to(a, ux + c_dx[k], uy + c_dy[k], uz + c_dz[k], qx, qy, qz);
        if (d >= rs) return;
        const int v = u + sh.off[k];
        if (!a.alive[v]) return;
        const int s = int(unsigned(ku));
        unsigned mb = __float_as_uint(d);
        const unsigned mu = unsigned(ku >> 32);
        if (mb < mu) mb = mu;
        if (mb < hi) {
          const unsigned long long cand = (static_cast<unsigned long long>(mb) << 32) | unsigned(s);
          const unsigned long long old = atomicMin(a.key + v, cand);
          if (old > cand) {
            if (old == BK_UNCLAIMED) touched[atomicAdd(&L->n_touch, 1)] = v;
            if (!(atomicOr(a.flags + v, kFront) & kFront)) nxt[atomicAdd(next_count, 1)] = v;
          }
        } else if (__ldcg(a.key + v) == BK_UNCLAIMED) {
          if (!(atomicOr(a.flags + v, kWaiting) & kWaiting)) far[atomicAdd(&L->n_far, 1)] = v;
        }
      };
      int lo, hi_i;
      if (own_share<C>(nc, kInvalStage, lo, hi_i)) {
        // step A: the round boundary's key of each frontier voxel, its mask, both positions and
        // the source's reach, in this CTA's shared memory
        unsigned long long *skey = reinterpret_cast<unsigned long long *>(stage_bytes());
        unsigned long long *spu = skey + kInvalStage, *sps = spu + kInvalStage;
        int *su = reinterpret_cast<int *>(sps + kInvalStage);
        unsigned *smask = reinterpret_cast<unsigned *>(su + kInvalStage);
        float *sreach = reinterpret_cast<float *>(smask + kInvalStage);
        for (int i = lo + int(threadIdx.x); i < hi_i; i += blockDim.x) {
          const int u = __ldcg(cur + i);
          const unsigned long long k = __ldcg(a.key + u);
          atomicAnd(a.flags + u, ~kFront);
          const int q = i - lo;
          su[q] = u;
          skey[q] = k;
          smask[q] = a.mask[u];
          sreach[q] = reach(a, int(unsigned(k)), sh.rscale, sh.rconst);
          int x, y, z;
          unravel3(u - sh.a0, sh.sx, sh.sy, x, y, z);
          spu[q] = pack3(x, y, z);
          unravel3(int(unsigned(k)) - sh.a0, sh.sx, sh.sy, x, y, z);
          sps[q] = pack3(x, y, z);
        }
        G::sync();
        for (int j = threadIdx.x; j < (hi_i - lo) * 26; j += blockDim.x) {
          const int q = j / 26, k = j - 26 * q;
          if (!((smask[q] >> k) & 1u)) continue;
          int ux, uy, uz, qx, qy, qz;
          unpack3(spu[q], ux, uy, uz);
          unpack3(sps[q], qx, qy, qz);
          offer(su[q], skey[q], k, ux, uy, uz, qx, qy, qz, sreach[q]);
        }
      } else {
        // step A: the round boundary's key of each frontier voxel, and both positions
        for (int i = G::tid(); i < nc; i += G::threads()) {
          const int u = __ldcg(cur + i);
          const unsigned long long k = __ldcg(a.key + u);
          atomicAnd(a.flags + u, ~kFront);
          wide[i] = k;
          int x, y, z;
          unravel3(u - sh.a0, sh.sx, sh.sy, x, y, z);
          side_u[i] = pack3(x, y, z);
          unravel3(int(unsigned(k)) - sh.a0, sh.sx, sh.sy, x, y, z);
          side_s[i] = pack3(x, y, z);
        }
        G::sync();
        for (long long j = G::tid(); j < (long long)nc * 32; j += G::threads()) {
          const int k = int(j & 31);
          if (k >= 26) continue;
          const int i = int(j >> 5);
          const int u = __ldcg(cur + i);
          if (!((a.mask[u] >> k) & 1u)) continue;
          const unsigned long long ku = __ldcg(wide + i);
          int ux, uy, uz, qx, qy, qz;
          unpack3(__ldcg(side_u + i), ux, uy, uz);
          unpack3(__ldcg(side_s + i), qx, qy, qz);
          offer(u, ku, k, ux, uy, uz, qx, qy, qz, reach(a, int(unsigned(ku)), sh.rscale, sh.rconst));
        }
      }
      G::sync();
    }
    const int nf = vload(&L->n_far);
    if (nf == 0) break;
    if (++work > bound) return false;
    // band boundary: every waiting voxel pulls the best offer of its claimed neighbours
    if (threadIdx.x == 0) sh.lowest = BK_INF_BITS;
    if (G::first()) L->n_keep = 0;
    // the offer of claimed neighbour key ku to waiting voxel c at (x, y, z), or ~0
    auto pull = [&](unsigned long long ku, int x, int y, int z) -> unsigned long long {
      const int s = int(unsigned(ku));
      int qx, qy, qz;
      unravel3(s - sh.a0, sh.sx, sh.sy, qx, qy, qz);
      const float d = distance_to(a, x, y, z, qx, qy, qz);
      if (d >= reach(a, s, sh.rscale, sh.rconst)) return ~0ull;
      unsigned mb = __float_as_uint(d);
      const unsigned mu = unsigned(ku >> 32);
      if (mb < mu) mb = mu;
      atomicMin(&sh.lowest, mb);
      return (static_cast<unsigned long long>(mb) << 32) | unsigned(s);
    };
    // claim the waiting voxel c with best offer b inside the new band, or keep it waiting
    auto settle = [&](int c, unsigned long long b, int *cur, int *cur_count) {
      if (b == kClaimedMark) return;
      if (b == BK_UNCLAIMED) { atomicAnd(a.flags + c, ~kWaiting); return; }
      if (unsigned(b >> 32) < hi) {
        a.key[c] = b;
        touched[atomicAdd(&L->n_touch, 1)] = c;
        atomicAnd(a.flags + c, ~kWaiting);
        atomicOr(a.flags + c, kFront);
        cur[atomicAdd(cur_count, 1)] = c;
      } else {
        keep[atomicAdd(&L->n_keep, 1)] = c;
      }
    };
    int lo, hi_f;
    if (own_share<C>(nf, kBandStage, lo, hi_f)) {
      // this CTA's waiting voxels in shared memory: nothing writes a key before the claims, which
      // come after a group barrier, so the pulls only wait for this CTA's staging
      unsigned long long *sbest = reinterpret_cast<unsigned long long *>(stage_bytes());
      unsigned long long *spc = sbest + kBandStage;
      int *sc = reinterpret_cast<int *>(spc + kBandStage);
      unsigned *smask = reinterpret_cast<unsigned *>(sc + kBandStage);
      for (int i = lo + int(threadIdx.x); i < hi_f; i += blockDim.x) {
        const int c = __ldcg(far + i);
        const int q = i - lo;
        sc[q] = c;
        sbest[q] = __ldcg(a.key + c) != BK_UNCLAIMED ? kClaimedMark : BK_UNCLAIMED;
        smask[q] = a.mask[c];
        int x, y, z;
        unravel3(c - sh.a0, sh.sx, sh.sy, x, y, z);
        spc[q] = pack3(x, y, z);
      }
      __syncthreads();
      for (int j = threadIdx.x; j < (hi_f - lo) * 26; j += blockDim.x) {
        const int q = j / 26, k = j - 26 * q;
        if (sbest[q] == kClaimedMark || !((smask[q] >> k) & 1u)) continue;
        const unsigned long long ku = __ldcg(a.key + sc[q] + sh.off[k]);
        if (ku == BK_UNCLAIMED) continue;
        int x, y, z;
        unpack3(spc[q], x, y, z);
        const unsigned long long o = pull(ku, x, y, z);
        if (o != ~0ull) atomicMin(sbest + q, o);
      }
      G::sync();
      const unsigned lowest = G::min_over(&sh.lowest);
      if (lowest != BK_INF_BITS) band = band_of(lowest, a.delta, band + 1);
      hi = __float_as_uint(__fmul_rn(float(band + 1), a.delta));
      int *cur = (r & 1) ? B : A;
      for (int i = lo + int(threadIdx.x); i < hi_f; i += blockDim.x) settle(sc[i - lo], sbest[i - lo], cur, &L->cnt[r % 3]);
    } else {
      for (int i = G::tid(); i < nf; i += G::threads()) {
        const int c = __ldcg(far + i);
        wide[i] = __ldcg(a.key + c) != BK_UNCLAIMED ? kClaimedMark : BK_UNCLAIMED;
        int x, y, z;
        unravel3(c - sh.a0, sh.sx, sh.sy, x, y, z);
        side_u[i] = pack3(x, y, z);
      }
      G::sync();
      for (long long j = G::tid(); j < (long long)nf * 32; j += G::threads()) {
        const int k = int(j & 31);
        if (k >= 26) continue;
        const int i = int(j >> 5);
        if (__ldcg(wide + i) == kClaimedMark) continue;
        const int c = __ldcg(far + i);
        if (!((a.mask[c] >> k) & 1u)) continue;
        const unsigned long long ku = __ldcg(a.key + c + sh.off[k]);
        if (ku == BK_UNCLAIMED) continue;
        int x, y, z;
        unpack3(__ldcg(side_u + i), x, y, z);
        const unsigned long long o = pull(ku, x, y, z);
        if (o != ~0ull) atomicMin(wide + i, o);
      }
      G::sync();
      const unsigned lowest = G::min_over(&sh.lowest);
      if (lowest != BK_INF_BITS) band = band_of(lowest, a.delta, band + 1);
      hi = __float_as_uint(__fmul_rn(float(band + 1), a.delta));
      int *cur = (r & 1) ? B : A;
      for (int i = G::tid(); i < nf; i += G::threads()) settle(__ldcg(far + i), __ldcg(wide + i), cur, &L->cnt[r % 3]);
    }
    G::sync();
    if (G::first()) L->n_far = L->n_keep;
    int *tmp = far; far = keep; keep = tmp;
    G::sync();
  }
  const int nt = vload(&L->n_touch);
  for (int i = G::tid(); i < nt; i += G::threads()) {
    const int v = __ldcg(touched + i);
    a.alive[v] = 0;
    a.key[v] = BK_UNCLAIMED;
    atomicAnd(a.flags + v, ~(kFront | kWaiting));
  }
  G::sync();
  return true;
}

template <int C>
__device__ void trace_loop(const EngineArgs &a, bool big) {
  using G = Group<C>;
  __shared__ Shared sh;
  __shared__ unsigned long long s_work[4];
  __shared__ unsigned long long s_prof[6];  // start, last lap, time in the four phases
  Shared *L = G::leader(&sh);
  if (threadIdx.x < 4) s_work[threadIdx.x] = 0;
  while (next_object<C>(a, sh, L, big)) {
    const int o = sh.obj;
    if (vload(&L->status) != kOk) {  // preparation failed; its status stands
      G::sync();
      continue;
    }
    int *L0 = a.lists + sh.begin, *L1 = L0 + a.F, *L2 = L1 + a.F, *L3 = L2 + a.F, *L4 = L3 + a.F;
    unsigned long long *wide = a.wide + sh.begin, *side_u = a.side + sh.begin, *side_s = a.side + a.F + sh.begin;
    int *store = a.store + a.store_begin[o];
    const long long store_cap = a.store_cap[o];
    int *rec_start = a.rec_start + a.rec_begin[o], *rec_len = a.rec_len + a.rec_begin[o];
    const long long rec_cap = a.rec_cap[o];
    const int mcount = a.manual_count[o];
    const int *manual = a.manual + a.manual_begin[o];
    const int acount = a.after_count[o];
    const int *after = a.after + a.after_begin[o];
    int after_used = 0;
    const int *order = a.order + sh.begin;
    const long long maxp = a.max_paths[o];
    long long paths = 0, used = 0;
    int cursor = 0;
    int status = kOk;
    // per-object phase timers, kept in shared memory by the first thread (registers are scarce)
    if (G::first()) {
      L->rounds = 0;
      s_prof[0] = s_prof[1] = now_ns();
      s_prof[2] = s_prof[3] = s_prof[4] = s_prof[5] = 0;
    }
    auto lap = [&](int phase) {
      if (G::first()) { const unsigned long long t = now_ns(); s_prof[2 + phase] += t - s_prof[1]; s_prof[1] = t; }
    };
    // The loop's steps, each with one flood: first the soma's ball (a soma: an invalidation from the
    // root with the soma's reach, trace.cu:199), then the parents' field (without fix_branching:
    // the object's SSSP from the root, kept until the object is done), then the paths. Every flood
    // function has this one call site, which keeps the kernel's registers for the paths' loop.
    if (threadIdx.x == 0) {
      sh.root = a.root[o];
      sh.soma_radius = a.soma_radius[o];
      sh.step = sh.soma_radius >= 0.0 ? 0 : (a.fix_branching ? 2 : 1);
      sh.skipped = 0;
    }
    __syncthreads();
    while (status == kOk) {
      const int step = sh.step;  // 0: the soma's ball, 1: the parents' field, 2: paths
      int t = -1, len = 1;
      bool ordered = false;  // t is the first alive voxel of the DAF order
      if (step == 2) {
        const long long taken = paths + sh.skipped;  // targets taken so far, empty paths included
        if (taken >= maxp) break;
        // the next target: manual targets first, then the first alive voxel of the order, then the
        // targets after (trace.cu:209-212)
        if (taken < mcount) {
          t = manual[taken];
          if (t < 0) t = a.target[o];  // the object's own target (the DAF argmax)
        } else {
          for (;;) {
            if (threadIdx.x == 0) sh.pos = INT32_MAX;
            G::sync();
            const int pos = cursor + G::tid();
            if (pos < sh.count && __ldcg(a.alive + order[pos])) atomicMin(&sh.pos, unsigned(pos));
            G::sync();
            const int found = int(G::min_over(&sh.pos));
            G::sync();
            if (found != INT32_MAX) { cursor = found; t = order[found]; ordered = true; break; }
            cursor += G::threads();
            if (cursor >= sh.count) { cursor = sh.count; break; }
          }
          if (t < 0 && after_used < acount) t = after[after_used++];
          if (t < 0) break;
        }
        lap(0);
      }
      if (step == 0) {
        if (G::first()) store[used] = sh.root;  // the ball's one source (the slot is reused)
        G::sync();
      } else if (step == 1 || a.fix_branching) {
        const unsigned long long rb = railroad<C>(a, sh, L, step == 1 ? sh.root : t, L0, L1, L2, L3, L4, wide);
        lap(1);
        if (vload(&L->status) != kOk) { status = vload(&L->status); break; }
        const int nt = vload(&L->n_touch);
        if (step == 1) {  // the parents' field stays; its queue flags are cleared now
          for (int i = G::tid(); i < nt; i += G::threads()) atomicAnd(a.flags + __ldcg(L4 + i), ~(kNearQueued | kFarQueued));
          if (G::first()) { s_work[0] += nt; s_work[1] += nt; }
          if (threadIdx.x == 0) sh.step = 2;  // every CTA of the group moves on (each has its own copy)
          G::sync();
          continue;
        }
        if (rb == BK_UNCLAIMED) {
          // No rail is reachable from t: an infinite penalty walls it off (a cavity the avocado
          // stage painted without refreshing the field). A target of the DAF order would be picked
          // again and again, so the object ends here (trace.cu:218-224); a manual target leaves an
          // empty path. Either way the flood's state goes back to rest first.
          for (int i = G::tid(); i < nt; i += G::threads()) {
            const int v = __ldcg(L4 + i);
            a.dist[v] = inf();
            atomicAnd(a.flags + v, ~(kNearQueued | kFarQueued));
          }
          if (G::first()) s_work[1] += nt;
          if (threadIdx.x == 0 && !ordered) sh.skipped += 1;  // every CTA keeps its own copy
          G::sync();
          if (ordered) break;
          continue;
        }
        // walk (one warp of the first CTA), then reset the flood's state over the voxels it touched
        if (G::rank() == 0 && threadIdx.x < 32) {
          const int n = backtrace(a, sh, rb, t, store + used, store_cap - used);
          if (threadIdx.x == 0) L->len = n;
        }
        G::sync();
        const float D = __uint_as_float(unsigned(rb >> 32));
        unsigned settled = 0;
        for (int i = G::tid(); i < nt; i += G::threads()) {
          const int v = __ldcg(L4 + i);
          settled += __ldcg(a.dist + v) <= D;
          a.dist[v] = inf();
          atomicAnd(a.flags + v, ~(kNearQueued | kFarQueued));
        }
        settled = __reduce_add_sync(kFull, settled);
        if ((threadIdx.x & 31) == 0) atomicAdd(&s_work[0], (unsigned long long)settled);
        if (G::first()) s_work[1] += nt;
        G::sync();
        lap(2);
      } else {  // the walk to the root through the parents' field
        if (G::rank() == 0 && threadIdx.x < 32) {
          const int n = parent_walk(a, sh, t, sh.root, store + used, store_cap - used);
          if (threadIdx.x == 0) L->len = n;
        }
        G::sync();
        lap(2);
      }
      if (step == 2) {
        len = vload(&L->len);
        if (sh.soma_radius >= 0.0 && len > 0) {
          if (G::rank() == 0 && threadIdx.x < 32) {
            const int n = soma_trim(a, sh, store + used, len, sh.root, sh.soma_radius, a.fix_branching != 0,
                                    store_cap - used);
            if (threadIdx.x == 0) L->len = n;
          }
          G::sync();
          len = vload(&L->len);
        }
        if (len < 0) { status = kStoreFull; break; }
        if (paths >= rec_cap) { status = kRecordsFull; break; }
      }
      const bool ball = step == 0;
      if (threadIdx.x == 0) {  // the reach of the invalidation's sources (the soma's for its ball)
        sh.rscale = ball ? a.soma_scale : a.scale;
        sh.rconst = ball ? a.soma_constant : a.constant;
      }
      __syncthreads();
      if (!invalidate<C>(a, sh, L, store + used, len, L0, L1, L2, L3, L4, wide, side_u, side_s)) {
        status = kBudget;
        break;
      }
      if (ball) {
        if (G::first()) s_work[2] += vload(&L->n_touch);
        if (threadIdx.x == 0) sh.step = a.fix_branching ? 2 : 1;  // every CTA of the group moves on
        G::sync();
        continue;
      }
      if (G::first()) { s_work[2] += vload(&L->n_touch); s_work[3] += 1; }
      lap(3);
      if (a.fix_branching)
        for (int i = G::tid(); i < len; i += G::threads()) a.pdrf[__ldcg(store + used + i)] = 0.0f;
      else
        for (int i = G::tid(); i < len; i += G::threads()) atomicOr(a.flags + __ldcg(store + used + i), kOnPath);
      if (G::first()) { rec_start[paths] = int(used); rec_len[paths] = len; }
      G::sync();
      used += len;
      ++paths;
    }
    if (!a.fix_branching) {  // the parents' field and the path marks go back to rest
      for (int i = G::tid(); i < sh.count; i += G::threads()) a.dist[a.vox[sh.begin + i]] = inf();
      for (long long i = G::tid(); i < used; i += G::threads()) atomicAnd(a.flags + __ldcg(store + i), ~kOnPath);
      G::sync();
    }
    if (G::first()) {
      a.status[o] = status;
      a.npaths[o] = int(paths);
      a.nstore[o] = int(used);
      unsigned long long *pr = a.profile + 8LL * o;
      pr[0] = s_prof[0]; pr[1] = now_ns();
      for (int q = 0; q < 4; ++q) pr[2 + q] = s_prof[2 + q];
      pr[6] = L->rounds & 0xFFFFFFFFull; pr[7] = L->rounds >> 32;
    }
    G::sync();
  }
  if (threadIdx.x < 4 && s_work[threadIdx.x]) atomicAdd(a.work + threadIdx.x, s_work[threadIdx.x]);
}

template <int C>
// The first a.lone_first clusters start on the small objects (each CTA alone, largest first) and
// then join the large ones; the others take the large objects first. So the longest lone-CTA
// objects run beside the clusters' objects from the start instead of after them.
__global__ void __launch_bounds__(kEngineThreads, kEngineCtasPerSm) trace_kernel(EngineArgs a) {
  if (int(blockIdx.x) / C < a.lone_first) {
    trace_loop<1>(a, false);
    trace_loop<C>(a, true);
  } else {
    trace_loop<C>(a, true);
    trace_loop<1>(a, false);
  }
}

cudaLaunchConfig_t cluster_config(int clusters, int ctas, cudaStream_t stream, cudaLaunchAttribute *attr) {
  cudaLaunchConfig_t config{};
  config.gridDim = dim3(unsigned(clusters * ctas));
  config.blockDim = dim3(kEngineThreads);
  config.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = unsigned(ctas);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  config.attrs = attr;
  config.numAttrs = 1;
  return config;
}

// Resident clusters of `kernel` on the current device (queried once per device and kernel: the
// query costs far more than a launch).
int resident_clusters(const void *kernel, int ctas, cudaStream_t stream) {
  static std::mutex lock;
  static std::map<std::pair<int, const void *>, int> known;
  int device = 0;
  BK_CUDA(cudaGetDevice(&device));
  std::lock_guard<std::mutex> guard(lock);
  auto it = known.find({device, kernel});
  if (it != known.end()) return it->second;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t probe = cluster_config(1, ctas, stream, attr);
  int cap = 1;
  BK_CUDA(cudaOccupancyMaxActiveClusters(&cap, kernel, &probe));
  known[{device, kernel}] = cap;
  return cap;
}

// As many clusters as are resident at once (no more than the work needs).
void launch(const void *kernel, int ctas, const EngineArgs &a, int nbig, cudaStream_t stream, int lone_percent = 0) {
  EngineArgs args = a;
  args.nbig = nbig;
  void *kargs[] = {&args};
  cudaLaunchAttribute attr[1];
  const int cap = std::max(1, resident_clusters(kernel, ctas, stream) * std::min(100, std::max(1, a.grid_percent)) / 100);
  const long long need = nbig + (a.nobj - nbig + ctas - 1) / ctas;
  const int clusters = int(std::max(1LL, std::min<long long>(cap, need)));
  args.lone_first = nbig < a.nobj ? clusters * lone_percent / 100 : 0;
  cudaLaunchConfig_t config = cluster_config(clusters, ctas, stream, attr);
  BK_CUDA(cudaLaunchKernelExC(&config, kernel, kargs));
}

}  // namespace

long long trace_cluster_voxels(long long foreground) {
  static std::mutex lock;
  static std::map<int, long long> known;  // resident engine CTAs per device
  int device = 0;
  BK_CUDA(cudaGetDevice(&device));
  long long ctas = 0;
  {
    std::lock_guard<std::mutex> guard(lock);
    auto it = known.find(device);
    if (it == known.end()) {
      int sms = 1, per_sm = 1;
      BK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
      BK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_kernel<kClusterCtas>, kEngineThreads, 0));
      it = known.emplace(device, std::max(1LL, (long long)sms * per_sm)).first;
    }
    ctas = it->second;
  }
  return std::max(kTraceClusterFloor, foreground / (2 * ctas));
}

int cluster_ctas(long long largest, long long foreground) {
  return largest * kWideClusterShare >= foreground ? kWideClusterCtas : kClusterCtas;
}

void launch_prepare(const EngineArgs &a, int nbig, int ctas, cudaStream_t stream) {
  if (ctas == kWideClusterCtas) launch((const void *)prepare_kernel<kWideClusterCtas>, ctas, a, nbig, stream);
  else launch((const void *)prepare_kernel<kClusterCtas>, kClusterCtas, a, nbig, stream);
}

void prepare_engine_launches(int prepare_ctas, int trace_ctas, cudaStream_t stream) {
  if (prepare_ctas == kWideClusterCtas) resident_clusters((const void *)prepare_kernel<kWideClusterCtas>, kWideClusterCtas, stream);
  else resident_clusters((const void *)prepare_kernel<kClusterCtas>, kClusterCtas, stream);
  if (trace_ctas == kWideClusterCtas) resident_clusters((const void *)trace_kernel<kWideClusterCtas>, kWideClusterCtas, stream);
  else resident_clusters((const void *)trace_kernel<kClusterCtas>, kClusterCtas, stream);
}

void launch_trace(const EngineArgs &a, int nbig, int ctas, int lone_percent, cudaStream_t stream) {
  if (ctas == kWideClusterCtas) launch((const void *)trace_kernel<kWideClusterCtas>, ctas, a, nbig, stream, lone_percent);
  else launch((const void *)trace_kernel<kClusterCtas>, kClusterCtas, a, nbig, stream, lone_percent);
}

}  // namespace bk
