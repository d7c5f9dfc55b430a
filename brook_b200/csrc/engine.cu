// Object engine kernels (see engine.hpp). Each CTA runs one object's chain; every flood round is
// "one warp per frontier voxel, one lane per neighbour" followed by a block barrier. State other
// lanes update with atomics (distances, keys, flags, liveness, rails) is always read through L2.
#include "common.cuh"
#include "engine.hpp"
#include "runtime.hpp"

namespace bk {
namespace {

constexpr int kWarps = kEngineThreads / 32;
constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr unsigned long long kMinFarNone = 0x7f8000007f800000ull;
constexpr unsigned long long kClaimedMark = 0xFFFFFFFFFFFFFFFEull;

struct Shared {
  int obj, begin, count, status;
  int a0, sx, sy, sz;  // the object's arena
  int n_cur, n_next, n_far, n_keep, n_touch, flag;
  unsigned lowest;
  float T;
  unsigned long long rb, minfar, best;
  int off[26];
  float w[26];
};

__device__ __forceinline__ float inf() { return __uint_as_float(BK_INF_BITS); }

__device__ __forceinline__ void unravel3(int i, int sx, int sy, int &x, int &y, int &z) {
  const int sxy = sx * sy;
  z = i / sxy;
  const int r = i - z * sxy;
  y = r / sx;
  x = r - y * sx;
}

// Minimum of a 64-bit value over the warp (two 32-bit reductions).
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
  const unsigned hi = __reduce_min_sync(kFull, unsigned(v >> 32));
  const unsigned lo = __reduce_min_sync(kFull, unsigned(v >> 32) == hi ? unsigned(v) : 0xFFFFFFFFu);
  return (static_cast<unsigned long long>(hi) << 32) | lo;
}

// Pulls the next object for this CTA and sets up its arena frame; false when the queue is empty.
__device__ bool next_object(const EngineArgs &a, Shared &sh) {
  if (threadIdx.x == 0) {
    const int j = atomicAdd(a.queue, 1);
    sh.obj = j < a.nobj ? a.schedule[j] : -1;
    if (sh.obj >= 0) {
      sh.begin = a.obj_begin[sh.obj];
      sh.count = a.obj_count[sh.obj];
      sh.status = kOk;
      const int r = a.obj_arena[sh.obj];
      sh.a0 = a.arena_offset[r];
      sh.sx = a.arena_dims[3 * r];
      sh.sy = a.arena_dims[3 * r + 1];
      sh.sz = a.arena_dims[3 * r + 2];
    }
  }
  __syncthreads();
  if (sh.obj >= 0 && threadIdx.x < 26) {
    const int k = threadIdx.x;
    sh.off[k] = c_dx[k] + sh.sx * (c_dy[k] + sh.sy * c_dz[k]);
    sh.w[k] = a.w[k];
  }
  __syncthreads();
  return sh.obj >= 0;
}

// ---------------------------------------------------------------------------------------------
// Geometric flood from `source` over the object's voxels into `d` (+inf at rest on them):
// Bellman-Ford rounds, fl(d[u] + w[k]). The fixed point is the least float32 path sum, which any
// schedule reaches. Returns false when the round bound is hit.
__device__ bool flood_geometric(const EngineArgs &a, Shared &sh, float *d, int source, int *A, int *B) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    d[source] = 0.0f;
    atomicOr(a.flags + source, kNearQueued);
    A[0] = source;
    sh.n_cur = 1;
    sh.n_next = 0;
  }
  __syncthreads();
  int *cur = A, *nxt = B;
  const long long bound = 8LL * sh.count + 256;
  for (long long round = 0;; ++round) {
    const int nc = sh.n_cur;
    if (nc == 0) break;
    if (round >= bound) return false;
    for (int i = warp; i < nc; i += kWarps) {
      int u = 0;
      float du = 0.0f;
      uint32_t m = 0;
      if (lane == 0) {
        u = __ldcg(cur + i);
        const unsigned was = atomicAnd(a.flags + u, ~kNearQueued);
        du = __ldcg(d + u + (was >> 30));
        m = a.mask[u];
      }
      u = __shfl_sync(kFull, u, 0);
      du = __shfl_sync(kFull, du, 0);
      m = __shfl_sync(kFull, m, 0);
      if (lane < 26 && ((m >> lane) & 1u)) {
        const int v = u + sh.off[lane];
        const float cand = __fadd_rn(du, sh.w[lane]);
        const float old = atomic_min_pos(d + v, cand);
        if (old > cand && !(atomicOr(a.flags + v, kNearQueued) & kNearQueued)) nxt[atomicAdd(&sh.n_next, 1)] = v;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) { sh.n_cur = sh.n_next; sh.n_next = 0; }
    int *t = cur; cur = nxt; nxt = t;
    __syncthreads();
  }
  return true;
}

// Largest finite value of `f` over the object's voxels, ties -> lowest flat index. Returns the
// packed key (value bits << 32 | ~flat), 0 when nothing is finite.
__device__ unsigned long long object_argmax(const EngineArgs &a, Shared &sh, const float *f) {
  if (threadIdx.x == 0) sh.best = 0;
  __syncthreads();
  unsigned long long best = 0;
  for (int i = threadIdx.x; i < sh.count; i += blockDim.x) {
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
  __syncthreads();
  const unsigned long long r = sh.best;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kEngineThreads) prepare_kernel(EngineArgs a) {
  __shared__ Shared sh;
  while (next_object(a, sh)) {
    const int o = sh.obj;
    int *A = a.lists + sh.begin, *B = a.lists + a.F + sh.begin;
    int root = a.border_root[o];
    if (root < 0) {
      // the farthest voxel (geometric distance) from the object's first voxel
      if (!flood_geometric(a, sh, a.daf, a.vox[sh.begin], A, B)) { if (threadIdx.x == 0) a.status[o] = kBudget; continue; }
      const unsigned long long k = object_argmax(a, sh, a.daf);
      root = int(0xFFFFFFFFu - unsigned(k));
      for (int i = threadIdx.x; i < sh.count; i += blockDim.x) a.daf[a.vox[sh.begin + i]] = inf();
      __syncthreads();
    }
    if (!flood_geometric(a, sh, a.daf, root, A, B)) { if (threadIdx.x == 0) a.status[o] = kBudget; continue; }
    const unsigned long long k = object_argmax(a, sh, a.daf);
    const float farthest = __uint_as_float(unsigned(k >> 32));
    const int target = int(0xFFFFFFFFu - unsigned(k));
    // PDRF of the object's voxels (the reference's pdrf_lab, batched_regular.inc:93-108):
    // (1 - dbf * M)^(2^squarings) * scale + daf * inv, one rounding per operation.
    const float M = a.M[o];
    const bool with_daf = farthest != 0.0f;
    const float inv = with_daf ? __double2float_rn(__ddiv_rn(1.0, (double)farthest)) : 0.0f;
    for (int i = threadIdx.x; i < sh.count; i += blockDim.x) {
      const int v = a.vox[sh.begin + i];
      float dv = a.dbf[v];
      if (dv == 0.0f) dv = inf();
      float p = __fsub_rn(1.0f, __fmul_rn(dv, M));
      for (int s = 0; s < a.squarings; ++s) p = __fmul_rn(p, p);
      p = __fmul_rn(p, a.pdrf_scale);
      if (with_daf) {
        float dd = __ldcg(a.daf + v);
        if (isinf(dd)) dd = 0.0f;
        p = __fadd_rn(p, __fmul_rn(dd, inv));
      }
      a.pdrf[v] = p;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      a.pdrf[root] = 0.0f;  // the root is the first rail
      a.root[o] = root;
      a.target[o] = target;
      a.max_daf[o] = farthest;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------------
// Railroad flood from target t over the object's voxels: entering v costs pdrf[v] (vw_step), rails
// (pdrf == 0) absorb. Near-far bands: the near band [.., T] is relaxed to convergence, bounded by
// the best rail found so far; the next band starts at the nearest deferred voxel. Returns the
// nearest rail as (distance bits << 32 | flat), BK_UNCLAIMED when no rail is reachable, and
// sets sh.status on a bound. The result is schedule-independent: every voxel at distance <= D
// (the nearest rail's) is exact when the flood stops.
__device__ unsigned long long railroad(const EngineArgs &a, Shared &sh, int t, int *A, int *B, int *FA, int *FB,
                                       int *touched) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    sh.n_touch = 1;
    touched[0] = t;
    sh.rb = BK_UNCLAIMED;
    sh.minfar = kMinFarNone;
    sh.n_cur = 0; sh.n_next = 0; sh.n_far = 0; sh.n_keep = 0;
    a.dist[t] = 0.0f;
    const float ft = __ldcg(a.pdrf + t);
    if (ft == 0.0f) sh.rb = static_cast<unsigned long long>(unsigned(t));
    else {
      A[0] = t;
      sh.n_cur = 1;
      atomicOr(a.flags + t, kNearQueued);
      sh.T = fmaxf(__fmul_rn(2.0f, ft), 1e-30f);
    }
  }
  __syncthreads();
  if (sh.rb != BK_UNCLAIMED) return sh.rb;
  int *cur = A, *nxt = B, *far = FA, *keep = FB;
  const long long bound = 16LL * sh.count + 256;
  long long work = 0;
  for (;;) {
    for (;;) {
      const int nc = sh.n_cur;
      if (nc == 0) break;
      if (++work > bound) { if (threadIdx.x == 0) sh.status = kBudget; __syncthreads(); return BK_UNCLAIMED; }
      const float T = sh.T;
      for (int i = warp; i < nc; i += kWarps) {
        int u = 0;
        float du = -1.0f, Tb = 0.0f;
        uint32_t m = 0;
        if (lane == 0) {
          u = __ldcg(cur + i);
          const unsigned was = atomicAnd(a.flags + u, ~kNearQueued);
          const float fu = __ldcg(a.pdrf + u);
          const float d = __ldcg(a.dist + u + (was >> 30));
          const unsigned long long rb = *(volatile unsigned long long *)&sh.rb;
          Tb = rb != BK_UNCLAIMED ? fminf(T, __uint_as_float(unsigned(rb >> 32))) : T;
          if (fu != 0.0f && d <= Tb) { du = d; m = a.mask[u]; }
        }
        du = __shfl_sync(kFull, du, 0);
        if (du < 0.0f) continue;
        u = __shfl_sync(kFull, u, 0);
        m = __shfl_sync(kFull, m, 0);
        Tb = __shfl_sync(kFull, Tb, 0);
        if (lane < 26 && ((m >> lane) & 1u)) {
          const int v = u + sh.off[lane];
          const float fv = __ldcg(a.pdrf + v);
          const float cand = vw_step(du, fv);
          const float old = atomic_min_pos(a.dist + v, cand);
          if (old > cand) {
            if (old == inf()) touched[atomicAdd(&sh.n_touch, 1)] = v;
            if (fv == 0.0f)
              atomicMin(&sh.rb, (static_cast<unsigned long long>(__float_as_uint(cand)) << 32) | unsigned(v));
            if (cand <= Tb) {
              if (!(atomicOr(a.flags + v, kNearQueued) & kNearQueued)) nxt[atomicAdd(&sh.n_next, 1)] = v;
            } else {
              atomicMin(&sh.minfar, (static_cast<unsigned long long>(__float_as_uint(cand)) << 32) | __float_as_uint(fv));
              if (!(atomicOr(a.flags + v, kFarQueued) & kFarQueued)) far[atomicAdd(&sh.n_far, 1)] = v;
            }
          }
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) { sh.n_cur = sh.n_next; sh.n_next = 0; }
      int *tmp = cur; cur = nxt; nxt = tmp;
      __syncthreads();
    }
    // band end: the nearest rail is final once it lies inside the band
    if (threadIdx.x == 0) {
      sh.flag = 0;
      if (sh.rb != BK_UNCLAIMED && __uint_as_float(unsigned(sh.rb >> 32)) <= sh.T) sh.flag = 1;
      else if (sh.minfar == kMinFarNone) sh.flag = 2;
      else {
        const float d = __uint_as_float(unsigned(sh.minfar >> 32)), f = __uint_as_float(unsigned(sh.minfar));
        float w = __fmul_rn(2.0f, f);
        const float lo = __fmul_rn(5e-4f, d);
        if (!(w > lo)) w = lo;
        sh.T = __fadd_rn(d, w);
        sh.minfar = kMinFarNone;
      }
      sh.n_keep = 0;
    }
    __syncthreads();
    if (sh.flag) return sh.flag == 1 ? sh.rb : BK_UNCLAIMED;
    // promote deferred voxels inside the new band
    const int nf = sh.n_far;
    const unsigned long long rb = sh.rb;
    const float Tp = rb != BK_UNCLAIMED ? fminf(sh.T, __uint_as_float(unsigned(rb >> 32))) : sh.T;
    for (int i = threadIdx.x; i < nf; i += blockDim.x) {
      const int w = __ldcg(far + i);
      const float dw = __ldcg(a.dist + w);
      if (dw <= Tp) {
        atomicAnd(a.flags + w, ~kFarQueued);
        if (!(atomicOr(a.flags + w, kNearQueued) & kNearQueued)) cur[atomicAdd(&sh.n_cur, 1)] = w;
      } else {
        atomicMin(&sh.minfar, (static_cast<unsigned long long>(__float_as_uint(dw)) << 32) | __float_as_uint(__ldcg(a.pdrf + w)));
        keep[atomicAdd(&sh.n_keep, 1)] = w;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) sh.n_far = sh.n_keep;
    int *tmp = far; far = keep; keep = tmp;
    __syncthreads();
  }
}

// Warp 0 walks from the nearest rail back to the target: the step goes to the neighbour of least
// distance (non-rail, lowest neighbour index among ties); at the first step the rail end is
// re-picked as the last road voxel's first rail in dijkstra3d order (lockstep_regular.inc:61-155).
// Writes the path target-first to out and returns its length (-1: no room).
__device__ int backtrace(const EngineArgs &a, Shared &sh, unsigned long long rb, int t, int *out, long long room) {
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
        if (__ldcg(a.pdrf + u) != 0.0f) db = __float_as_uint(__ldcg(a.dist + u));
      }
      const unsigned mb = __reduce_min_sync(kFull, db);
      if (mb < BK_INF_BITS) kb = int(__reduce_min_sync(kFull, db == mb ? unsigned(lane) : 64u));
    }
    if (step == 0 && kb >= 0) {
      const int u = cur + sh.off[kb];
      const uint32_t mu = a.mask[u];
      unsigned key = 64;
      if (lane < 26 && ((mu >> lane) & 1u) && __ldcg(a.pdrf + u + sh.off[lane]) == 0.0f) key = unsigned(c_d3rank[lane]);
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

__device__ __forceinline__ float straight(const EngineArgs &a, const Shared &sh, int x, int y, int z, int s) {
  int qx, qy, qz;
  unravel3(s - sh.a0, sh.sx, sh.sy, qx, qy, qz);
  const float dx = __fmul_rn(a.wx, float(x - qx)), dy = __fmul_rn(a.wy, float(y - qy)), dz = __fmul_rn(a.wz, float(z - qz));
  return sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}
__device__ __forceinline__ float reach(const EngineArgs &a, int s) {
  return __fadd_rn(__fmul_rn(a.scale, a.dbf[s]), a.constant);
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
__device__ bool invalidate(const EngineArgs &a, Shared &sh, const int *path, int npath, int *A, int *B, int *FA,
                           int *FB, int *touched, unsigned long long *wide) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) { sh.n_cur = 0; sh.n_next = 0; sh.n_far = 0; sh.n_keep = 0; sh.n_touch = 0; }
  __syncthreads();
  for (int i = threadIdx.x; i < npath; i += blockDim.x) {
    const int p = path[i];
    if (!__ldcg(a.alive + p)) continue;
    const unsigned long long old = atomicMin(a.key + p, static_cast<unsigned long long>(unsigned(p)));
    if (old == BK_UNCLAIMED) {
      atomicOr(a.flags + p, kFront);
      A[atomicAdd(&sh.n_cur, 1)] = p;
      touched[atomicAdd(&sh.n_touch, 1)] = p;
    }
  }
  __syncthreads();
  int *cur = A, *nxt = B, *far = FA, *keep = FB;
  const long long bound = 64LL * sh.count + 1024;
  long long work = 0;
  int band = 0;
  for (;;) {
    unsigned hi = __float_as_uint(__fmul_rn(float(band + 1), a.delta));
    for (;;) {
      const int nc = sh.n_cur;
      if (nc == 0) break;
      if (++work > bound) return false;
      for (int i = threadIdx.x; i < nc; i += blockDim.x) {  // the round boundary's keys
        const int u = __ldcg(cur + i);
        wide[i] = __ldcg(a.key + u);
        atomicAnd(a.flags + u, ~kFront);
      }
      __syncthreads();
      for (int i = warp; i < nc; i += kWarps) {
        int u = 0, s = 0, ux = 0, uy = 0, uz = 0, qx = 0, qy = 0, qz = 0;
        unsigned mu = 0;
        uint32_t m = 0;
        float R = 0.0f;
        if (lane == 0) {
          u = __ldcg(cur + i);
          const unsigned long long k = __ldcg(wide + i);
          s = int(unsigned(k));
          mu = unsigned(k >> 32);
          m = a.mask[u];
          R = reach(a, s);
          unravel3(u - sh.a0, sh.sx, sh.sy, ux, uy, uz);
          unravel3(s - sh.a0, sh.sx, sh.sy, qx, qy, qz);
        }
        u = __shfl_sync(kFull, u, 0); s = __shfl_sync(kFull, s, 0); mu = __shfl_sync(kFull, mu, 0);
        m = __shfl_sync(kFull, m, 0); R = __shfl_sync(kFull, R, 0);
        ux = __shfl_sync(kFull, ux, 0); uy = __shfl_sync(kFull, uy, 0); uz = __shfl_sync(kFull, uz, 0);
        qx = __shfl_sync(kFull, qx, 0); qy = __shfl_sync(kFull, qy, 0); qz = __shfl_sync(kFull, qz, 0);
        if (lane >= 26 || !((m >> lane) & 1u)) continue;
        const int v = u + sh.off[lane];
        if (!__ldcg(a.alive + v)) continue;
        const float dx = __fmul_rn(a.wx, float(ux + c_dx[lane] - qx));
        const float dy = __fmul_rn(a.wy, float(uy + c_dy[lane] - qy));
        const float dz = __fmul_rn(a.wz, float(uz + c_dz[lane] - qz));
        const float d = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
        if (d >= R) continue;
        unsigned mb = __float_as_uint(d);
        if (mb < mu) mb = mu;
        if (mb < hi) {
          const unsigned long long cand = (static_cast<unsigned long long>(mb) << 32) | unsigned(s);
          const unsigned long long old = atomicMin(a.key + v, cand);
          if (old > cand) {
            if (old == BK_UNCLAIMED) touched[atomicAdd(&sh.n_touch, 1)] = v;
            if (!(atomicOr(a.flags + v, kFront) & kFront)) nxt[atomicAdd(&sh.n_next, 1)] = v;
          }
        } else if (__ldcg(a.key + v) == BK_UNCLAIMED) {
          if (!(atomicOr(a.flags + v, kWaiting) & kWaiting)) far[atomicAdd(&sh.n_far, 1)] = v;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) { sh.n_cur = sh.n_next; sh.n_next = 0; }
      int *tmp = cur; cur = nxt; nxt = tmp;
      __syncthreads();
    }
    const int nf = sh.n_far;
    if (nf == 0) break;
    if (++work > bound) return false;
    // band boundary: every waiting voxel pulls the best offer of its claimed neighbours
    if (threadIdx.x == 0) { sh.lowest = BK_INF_BITS; sh.n_keep = 0; }
    __syncthreads();
    for (int i = warp; i < nf; i += kWarps) {
      int c = 0;
      unsigned long long kc = 0;
      if (lane == 0) { c = __ldcg(far + i); kc = __ldcg(a.key + c); }
      c = __shfl_sync(kFull, c, 0);
      kc = __shfl_sync(kFull, kc, 0);
      if (kc != BK_UNCLAIMED) { if (lane == 0) wide[i] = kClaimedMark; continue; }
      const uint32_t m = a.mask[c];
      unsigned long long best = BK_UNCLAIMED;
      if (lane < 26 && ((m >> lane) & 1u)) {
        const unsigned long long ku = __ldcg(a.key + c + sh.off[lane]);
        if (ku != BK_UNCLAIMED) {
          const int s = int(unsigned(ku));
          int x, y, z;
          unravel3(c - sh.a0, sh.sx, sh.sy, x, y, z);
          const float d = straight(a, sh, x, y, z, s);
          if (d < reach(a, s)) {
            unsigned mb = __float_as_uint(d);
            const unsigned mu = unsigned(ku >> 32);
            if (mb < mu) mb = mu;
            best = (static_cast<unsigned long long>(mb) << 32) | unsigned(s);
          }
        }
      }
      best = warp_min_u64(best);
      if (lane == 0) {
        wide[i] = best;
        if (best != BK_UNCLAIMED) atomicMin(&sh.lowest, unsigned(best >> 32));
      }
    }
    __syncthreads();
    if (sh.lowest != BK_INF_BITS) band = band_of(sh.lowest, a.delta, band + 1);
    hi = __float_as_uint(__fmul_rn(float(band + 1), a.delta));
    for (int i = threadIdx.x; i < nf; i += blockDim.x) {
      const int c = __ldcg(far + i);
      const unsigned long long b = __ldcg(wide + i);
      if (b == kClaimedMark) continue;
      if (b == BK_UNCLAIMED) { atomicAnd(a.flags + c, ~kWaiting); continue; }
      if (unsigned(b >> 32) < hi) {
        a.key[c] = b;
        touched[atomicAdd(&sh.n_touch, 1)] = c;
        atomicAnd(a.flags + c, ~kWaiting);
        atomicOr(a.flags + c, kFront);
        cur[atomicAdd(&sh.n_cur, 1)] = c;
      } else {
        keep[atomicAdd(&sh.n_keep, 1)] = c;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) sh.n_far = sh.n_keep;
    int *tmp = far; far = keep; keep = tmp;
    __syncthreads();
  }
  const int nt = sh.n_touch;
  for (int i = threadIdx.x; i < nt; i += blockDim.x) {
    const int v = __ldcg(touched + i);
    a.alive[v] = 0;
    a.key[v] = BK_UNCLAIMED;
    atomicAnd(a.flags + v, ~(kFront | kWaiting));
  }
  __syncthreads();
  return true;
}

__global__ void __launch_bounds__(kEngineThreads) trace_kernel(EngineArgs a) {
  __shared__ Shared sh;
  __shared__ int s_pos;
  __shared__ unsigned long long s_work[4];
  if (threadIdx.x < 4) s_work[threadIdx.x] = 0;
  while (next_object(a, sh)) {
    const int o = sh.obj;
    int *L0 = a.lists + sh.begin, *L1 = L0 + a.F, *L2 = L1 + a.F, *L3 = L2 + a.F, *L4 = L3 + a.F;
    unsigned long long *wide = a.wide + sh.begin;
    int *store = a.store + a.store_begin[o];
    const long long store_cap = a.store_cap[o];
    int *rec_start = a.rec_start + a.rec_begin[o], *rec_len = a.rec_len + a.rec_begin[o];
    const long long rec_cap = a.rec_cap[o];
    const int mcount = a.manual_count[o];
    const int *manual = a.manual + a.manual_begin[o];
    const int *order = a.order + sh.begin;
    const long long maxp = a.max_paths[o];
    long long paths = 0, used = 0;
    int cursor = 0;
    int status = kOk;
    while (paths < maxp) {
      // the next target: manual targets first, then the first alive voxel of the order
      int t = -1;
      if (paths < mcount) {
        t = manual[paths];
        if (t < 0) t = a.target[o];  // the object's own target (the DAF argmax)
      } else {
        for (;;) {
          if (threadIdx.x == 0) s_pos = INT32_MAX;
          __syncthreads();
          const int pos = cursor + threadIdx.x;
          if (pos < sh.count && __ldcg(a.alive + order[pos])) atomicMin(&s_pos, pos);
          __syncthreads();
          const int found = s_pos;
          __syncthreads();
          if (found != INT32_MAX) { cursor = found; t = order[found]; break; }
          cursor += blockDim.x;
          if (cursor >= sh.count) { cursor = sh.count; break; }
        }
        if (t < 0) break;
      }
      const unsigned long long rb = railroad(a, sh, t, L0, L1, L2, L3, L4);
      if (sh.status != kOk) { status = sh.status; break; }
      if (rb == BK_UNCLAIMED) { status = kNoRail; break; }
      // walk (warp 0), then reset the flood's state over the voxels it touched
      if (threadIdx.x < 32) {
        const int len = backtrace(a, sh, rb, t, store + used, store_cap - used);
        if (threadIdx.x == 0) s_pos = len;
      }
      __syncthreads();
      const int len = s_pos;
      const int nt = sh.n_touch;
      const float D = __uint_as_float(unsigned(rb >> 32));
      unsigned settled = 0;
      for (int i = threadIdx.x; i < nt; i += blockDim.x) {
        const int v = __ldcg(L4 + i);
        settled += __ldcg(a.dist + v) <= D;
        a.dist[v] = inf();
        atomicAnd(a.flags + v, ~(kNearQueued | kFarQueued));
      }
      settled = __reduce_add_sync(0xFFFFFFFFu, settled);
      if ((threadIdx.x & 31) == 0) atomicAdd(&s_work[0], (unsigned long long)settled);
      if (threadIdx.x == 0) s_work[1] += nt;
      __syncthreads();
      if (len < 0) { status = kStoreFull; break; }
      if (paths >= rec_cap) { status = kRecordsFull; break; }
      if (!invalidate(a, sh, store + used, len, L0, L1, L2, L3, L4, wide)) { status = kBudget; break; }
      if (threadIdx.x == 0) { s_work[2] += sh.n_touch; s_work[3] += 1; }
      for (int i = threadIdx.x; i < len; i += blockDim.x) a.pdrf[store[used + i]] = 0.0f;
      if (threadIdx.x == 0) { rec_start[paths] = int(used); rec_len[paths] = len; }
      __syncthreads();
      used += len;
      ++paths;
    }
    if (threadIdx.x == 0) {
      a.status[o] = status;
      a.npaths[o] = int(paths);
      a.nstore[o] = int(used);
    }
    __syncthreads();
  }
  if (threadIdx.x < 4 && s_work[threadIdx.x]) atomicAdd(a.work + threadIdx.x, s_work[threadIdx.x]);
}

}  // namespace

int engine_grid(int sm_count, int nobj, bool trace) {
  int per_sm = 1;
  BK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace ? (const void *)trace_kernel : (const void *)prepare_kernel,
                                                        kEngineThreads, 0));
  per_sm = per_sm < 1 ? 1 : per_sm;
  const int full = sm_count * per_sm;
  return nobj < full ? (nobj < 1 ? 1 : nobj) : full;
}

void launch_prepare(const EngineArgs &a, int grid, cudaStream_t stream) {
  prepare_kernel<<<grid, kEngineThreads, 0, stream>>>(a);
  BK_CUDA(cudaGetLastError());
}

void launch_trace(const EngineArgs &a, int grid, cudaStream_t stream) {
  trace_kernel<<<grid, kEngineThreads, 0, stream>>>(a);
  BK_CUDA(cudaGetLastError());
}

}  // namespace bk
