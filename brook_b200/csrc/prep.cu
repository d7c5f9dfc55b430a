// Preamble kernels: per-component boxes and counts, the neighbour masks every later stage steps
// through, per-component maxima, fills and face extraction.
#include <algorithm>

#include "common.cuh"
#include "kernels.hpp"

namespace bk {
namespace {

// Boxes and counts in one pass (the reference's analyze, preamble.cu:10-29). A block takes
// kChunk consecutive voxels (each warp 32 at a time, coalesced); a warp's voxels of one id are
// reduced with match + redux (count, low and high x, y, z) and merged into the block's table of
// kSlots ids in shared memory; the table then goes to the global boxes with one guarded atomic
// per field and id (an id the table cannot take goes there directly). Dense volumes hold a few ids
// per chunk, so the global atomics fall from one per row run to one per chunk.
constexpr int kChunk = 2048, kSlots = 64;

__device__ __forceinline__ int table_slot(uint32_t *keys, uint32_t id) {
  int h = int((id * 0x9E3779B1u) >> 26);  // kSlots = 64
  for (int probe = 0; probe < kSlots; ++probe, h = (h + 1) & (kSlots - 1)) {
    const uint32_t k = keys[h];
    if (k == id) return h;
    if (k == 0) {
      const uint32_t prev = atomicCAS(keys + h, 0u, id);
      if (prev == 0u || prev == id) return h;
    }
  }
  return -1;
}

__device__ __forceinline__ void box_update(int *l, int *h, unsigned long long *count, const int lo[3], const int hi[3],
                                           unsigned n) {
  atomicAdd(count, (unsigned long long)n);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (__ldcg(l + a) > lo[a]) atomicMin(l + a, lo[a]);
    if (__ldcg(h + a) < hi[a]) atomicMax(h + a, hi[a]);
  }
}

__global__ void __launch_bounds__(256) analyze_kernel(const uint32_t *__restrict__ ids, Dims d, int *lo, int *hi,
                                                      unsigned long long *counts) {
  __shared__ uint32_t keys[kSlots];
  __shared__ unsigned cnt[kSlots];
  __shared__ int slo[kSlots][3], shi[kSlots][3];
  for (int t = threadIdx.x; t < kSlots; t += blockDim.x) {
    keys[t] = 0;
    cnt[t] = 0;
    for (int a = 0; a < 3; ++a) { slo[t][a] = INT32_MAX; shi[t][a] = -1; }
  }
  __syncthreads();
  const long long n = d.n(), begin = (long long)blockIdx.x * kChunk;
  const int lane = threadIdx.x & 31;
  for (long long i = begin + threadIdx.x; i < begin + kChunk; i += blockDim.x) {  // warp-uniform bounds
    const bool in = i < n;
    const uint32_t id = in ? ids[i] : 0u;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, id);
    // the warp's first voxel's position; when the 32 voxels lie in one row (the usual case), an
    // id's extent along x comes from its lanes and y, z are the row's
    int x0 = 0, y0 = 0, z0 = 0;
    if (lane == 0 && in) unravel((int)i, d, x0, y0, z0);
    x0 = __shfl_sync(0xFFFFFFFFu, x0, 0);
    y0 = __shfl_sync(0xFFFFFFFFu, y0, 0);
    z0 = __shfl_sync(0xFFFFFFFFu, z0, 0);
    const bool one_row = x0 + 31 < d.sx && i - lane + 31 < n;  // warp-uniform
    int l3[3], h3[3];
    if (one_row) {
      l3[0] = x0 + __ffs(peers) - 1;
      h3[0] = x0 + 31 - __clz(peers);
      l3[1] = h3[1] = y0;
      l3[2] = h3[2] = z0;
    } else {
      int x = 0, y = 0, z = 0;
      if (in) unravel((int)i, d, x, y, z);
      l3[0] = int(__reduce_min_sync(peers, unsigned(x)));
      h3[0] = int(__reduce_max_sync(peers, unsigned(x)));
      l3[1] = int(__reduce_min_sync(peers, unsigned(y)));
      h3[1] = int(__reduce_max_sync(peers, unsigned(y)));
      l3[2] = int(__reduce_min_sync(peers, unsigned(z)));
      h3[2] = int(__reduce_max_sync(peers, unsigned(z)));
    }
    if (id == 0 || lane != __ffs(peers) - 1) continue;
    const int slot = table_slot(keys, id);
    if (slot < 0) {
      box_update(lo + 3 * (long long)id, hi + 3 * (long long)id, counts + id, l3, h3, __popc(peers));
      continue;
    }
    atomicAdd(cnt + slot, unsigned(__popc(peers)));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      atomicMin(&slo[slot][a], l3[a]);
      atomicMax(&shi[slot][a], h3[a]);
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kSlots; t += blockDim.x) {
    const uint32_t id = keys[t];
    if (id) box_update(lo + 3 * (long long)id, hi + 3 * (long long)id, counts + id, slo[t], shi[t], cnt[t]);
  }
}

// The mask of a column of 32x8 voxels and kMaskZ planes. The block streams the column's halo
// planes (34x10 ids each, 0 outside the volume, which no voxel's id equals) through a ring of
// kRing shared-memory planes with asynchronous copies (cp.async, zero-filled outside), up to
// kRing - 2 planes ahead of the plane it reads; each thread holds the 3x3 neighbourhoods of three planes
// in registers, so a voxel costs nine shared loads (of the plane ahead) and 26 register compares.
// Vec: rows of a multiple of four ids at a 16-byte aligned base, copied in 16-byte pieces from
// x0 - 4 (ten per row); otherwise one 4-byte copy per id. Block (32, 8) threads, grid (x blocks,
// y blocks, z blocks).
constexpr int kMaskX = 32, kMaskY = 8, kMaskZ = 32, kRing = 8;
constexpr int kRowWords = kMaskX + 8, kPlaneWords = kRowWords * (kMaskY + 2);  // a row holds x0 - 4 .. x0 + 35

__device__ __forceinline__ void copy_async(uint32_t *dst, const uint32_t *src, int bytes, bool in) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(in ? 16 : 0) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(in ? 4 : 0) : "memory");
}

template <bool Vec>
__device__ __forceinline__ void mask_plane_copy(uint32_t *slot, const uint32_t *__restrict__ ids, const Dims &d,
                                                int x0, int y0, int z) {
  const int t = threadIdx.x + kMaskX * threadIdx.y;
  const bool zin = z >= 0 && z < d.sz;
  if (Vec) {
    if (t >= 10 * (kMaskY + 2)) return;
    const int row = t / 10, x = x0 - 4 + 4 * (t % 10), y = y0 + row - 1;
    const bool in = zin && y >= 0 && y < d.sy && x >= 0 && x < d.sx;
    const uint32_t *src = in ? ids + (x + (long long)d.sx * (y + (long long)d.sy * z)) : ids;
    copy_async(slot + row * kRowWords + 4 * (t % 10), src, 16, in);
  } else {
    for (int q = t; q < (kMaskX + 2) * (kMaskY + 2); q += kMaskX * kMaskY) {
      const int row = q / (kMaskX + 2), c = q % (kMaskX + 2), x = x0 - 1 + c, y = y0 + row - 1;
      const bool in = zin && y >= 0 && y < d.sy && x >= 0 && x < d.sx;
      const uint32_t *src = in ? ids + (x + (long long)d.sx * (y + (long long)d.sy * z)) : ids;
      copy_async(slot + row * kRowWords + 3 + c, src, 4, in);
    }
  }
}

template <bool Vec>
__global__ void __launch_bounds__(kMaskX * kMaskY, 4) mask_kernel(const uint32_t *__restrict__ ids, Dims d,
                                                                 uint32_t *__restrict__ mask) {
  constexpr int8_t DX[26] = {BK_NEIGHBOUR_DX}, DY[26] = {BK_NEIGHBOUR_DY}, DZ[26] = {BK_NEIGHBOUR_DZ};
  __shared__ __align__(16) uint32_t ring[kRing * kPlaneWords];
  const int x0 = blockIdx.x * kMaskX, y0 = blockIdx.y * kMaskY, z0 = blockIdx.z * kMaskZ;
  const int planes = min(kMaskZ, d.sz - z0) + 2;  // halo planes hz = 0 .. planes - 1 are z0 - 1 + hz
  // halo plane hz lives in slot hz % kRing; one commit group per plane index, empty past the end
  auto issue = [&](int hz) {
    if (hz < planes) mask_plane_copy<Vec>(ring + (hz % kRing) * kPlaneWords, ids, d, x0, y0, z0 - 1 + hz);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
#pragma unroll
  for (int hz = 0; hz < kRing; ++hz) issue(hz);
  asm volatile("cp.async.wait_group %0;\n" ::"n"(kRing - 2) : "memory");  // planes 0 and 1
  __syncthreads();
  const int lane = threadIdx.x, x = x0 + lane, y = y0 + threadIdx.y;
  const int col = 3 + lane + kRowWords * threadIdx.y;  // the (-1, -1) corner of this column's 3x3
  uint32_t w[3][9];                                    // planes z - 1, z, z + 1; index (dy + 1) * 3 + dx + 1
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int j = 0; j < 9; ++j) w[p][j] = ring[p * kPlaneWords + col + j % 3 + kRowWords * (j / 3)];
  const bool mine = x < d.sx && y < d.sy;
  for (int lz = 0; lz + 2 < planes; ++lz) {  // block-uniform trip count
    // groups issued: planes 0 .. lz + kRing - 1; plane lz + 2 must have landed
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kRing - 3) : "memory");
    __syncthreads();  // every copy of plane lz + 2 landed; plane lz (read two steps ago) is free
    issue(lz + kRing);
    const uint32_t *next = ring + ((lz + 2) % kRing) * kPlaneWords + col;
#pragma unroll
    for (int j = 0; j < 9; ++j) w[2][j] = next[j % 3 + kRowWords * (j / 3)];
    const uint32_t id = w[1][4];
    uint32_t m = 0;
    if (id) {
#pragma unroll
      for (int k = 0; k < 26; ++k)
        if (w[1 + DZ[k]][(DY[k] + 1) * 3 + DX[k] + 1] == id) m |= 1u << k;
    }
    if (mine) mask[x + (long long)d.sx * (y + (long long)d.sy * (z0 + lz))] = m;
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      w[0][j] = w[1][j];
      w[1][j] = w[2][j];
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// Per id the largest finite field value (as float bits), by the same block tables as analyze:
// the warp's maximum of an id (match + redux), then the block's, then one guarded atomic per id
// and block.
__global__ void __launch_bounds__(256) segmax_kernel(const float *__restrict__ f, const uint32_t *__restrict__ ids,
                                                     long long n, unsigned *best) {
  __shared__ uint32_t keys[kSlots];
  __shared__ unsigned top[kSlots];
  for (int t = threadIdx.x; t < kSlots; t += blockDim.x) { keys[t] = 0; top[t] = 0; }
  __syncthreads();
  const long long begin = (long long)blockIdx.x * kChunk;
  const int lane = threadIdx.x & 31;
  for (long long i = begin + threadIdx.x; i < begin + kChunk; i += blockDim.x) {
    const bool in = i < n;
    const uint32_t id = in ? ids[i] : 0u;
    const float v = in ? f[i] : 0.0f;
    const unsigned bits = (id != 0 && v < __uint_as_float(BK_INF_BITS)) ? __float_as_uint(v) : 0u;
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, id);
    const unsigned m = __reduce_max_sync(peers, bits);  // the largest bits of this warp's voxels of the id
    if (id == 0 || lane != __ffs(peers) - 1) continue;
    const int slot = table_slot(keys, id);
    if (slot < 0) {
      if (__ldcg(best + id) < m) atomicMax(best + id, m);
    } else {
      atomicMax(top + slot, m);
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kSlots; t += blockDim.x) {
    const uint32_t id = keys[t];
    if (id && __ldcg(best + id) < top[t]) atomicMax(best + id, top[t]);
  }
}

// The same maxima four voxels to a thread, for 16-byte aligned fields and ids: one 16-byte load
// of each, then the thread merges its own runs of one id (a run's maximum, kept where the run
// starts) and the warp meets once per run position that some lane starts a run at. Inside rows
// the four voxels mostly share one id, so a warp of 128 voxels needs one match round where the
// scalar kernel needs four. Runs of id 0 or of maximum 0 change nothing and are skipped.
constexpr int kQuadChunk = 4096;

__global__ void __launch_bounds__(256) segmax4_kernel(const float *__restrict__ f, const uint32_t *__restrict__ ids,
                                                      long long n, unsigned *best) {
  __shared__ uint32_t keys[kSlots];
  __shared__ unsigned top[kSlots];
  for (int t = threadIdx.x; t < kSlots; t += blockDim.x) { keys[t] = 0; top[t] = 0; }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long begin = (long long)blockIdx.x * kQuadChunk;
#pragma unroll
  for (int it = 0; it < kQuadChunk / (4 * 256); ++it) {  // the same trip count on every lane
    const long long i = begin + 4LL * (it * 256 + threadIdx.x);
    uint32_t id[4];
    float v[4];
    if (i + 3 < n) {
      const uint4 q = *reinterpret_cast<const uint4 *>(ids + i);
      const float4 x = *reinterpret_cast<const float4 *>(f + i);
      id[0] = q.x; id[1] = q.y; id[2] = q.z; id[3] = q.w;
      v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        id[k] = i + k < n ? ids[i + k] : 0u;
        v[k] = i + k < n ? f[i + k] : 0.0f;
      }
    }
    unsigned run[4];  // run[k]: the maximum of the run of id[k] from voxel k to the thread's last
#pragma unroll
    for (int k = 3; k >= 0; --k) {
      const unsigned bits = (id[k] != 0 && v[k] < __uint_as_float(BK_INF_BITS)) ? __float_as_uint(v[k]) : 0u;
      run[k] = (k < 3 && id[k] == id[k + 1]) ? max(bits, run[k + 1]) : bits;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const bool has = (k == 0 || id[k] != id[k - 1]) && id[k] != 0 && run[k] != 0;
      if (!__any_sync(0xFFFFFFFFu, has)) continue;  // warp-uniform
      const uint32_t key = has ? id[k] : 0u;
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
      const unsigned m = __reduce_max_sync(peers, has ? run[k] : 0u);
      if (!has || lane != __ffs(peers) - 1) continue;
      const int slot = table_slot(keys, key);
      if (slot < 0) {
        if (__ldcg(best + key) < m) atomicMax(best + key, m);
      } else {
        atomicMax(top + slot, m);
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kSlots; t += blockDim.x) {
    const uint32_t id = keys[t];
    if (id && __ldcg(best + id) < top[t]) atomicMax(best + id, top[t]);
  }
}

// Boxes and counts four voxels to a thread, for 16-byte aligned ids in rows of a multiple of four
// voxels (so a thread's four voxels share y and z): the thread's runs of one id (start x, length)
// meet the warp's once per run position that some lane starts a run at, as in segmax4_kernel. When
// the warp's 128 voxels lie in one row, y and z are the row's and only x is reduced.
__global__ void __launch_bounds__(256) analyze4_kernel(const uint32_t *__restrict__ ids, Dims d, int *lo, int *hi,
                                                       unsigned long long *counts) {
  __shared__ uint32_t keys[kSlots];
  __shared__ unsigned cnt[kSlots];
  __shared__ int slo[kSlots][3], shi[kSlots][3];
  for (int t = threadIdx.x; t < kSlots; t += blockDim.x) {
    keys[t] = 0;
    cnt[t] = 0;
    for (int a = 0; a < 3; ++a) { slo[t][a] = INT32_MAX; shi[t][a] = -1; }
  }
  __syncthreads();
  const long long n = d.n(), begin = (long long)blockIdx.x * kQuadChunk;
  const int lane = threadIdx.x & 31;
#pragma unroll 1
  for (int it = 0; it < kQuadChunk / (4 * 256); ++it) {  // the same trip count on every lane
    const long long i = begin + 4LL * (it * 256 + threadIdx.x);
    uint32_t id[4];
    if (i + 3 < n) {
      const uint4 q = *reinterpret_cast<const uint4 *>(ids + i);
      id[0] = q.x; id[1] = q.y; id[2] = q.z; id[3] = q.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) id[k] = i + k < n ? ids[i + k] : 0u;
    }
    int x = 0, y = 0, z = 0;
    if (i < n) unravel((int)i, d, x, y, z);
    const int x0 = __shfl_sync(0xFFFFFFFFu, x, 0);
    const bool one_row = x0 + 127 < d.sx && i - 4 * lane + 127 < n;  // warp-uniform
    unsigned len[4];  // len[k]: the length of the run of id[k] from voxel k to the thread's last
#pragma unroll
    for (int k = 3; k >= 0; --k) len[k] = (k < 3 && id[k] == id[k + 1]) ? len[k + 1] + 1 : 1u;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const bool has = (k == 0 || id[k] != id[k - 1]) && id[k] != 0;
      if (!__any_sync(0xFFFFFFFFu, has)) continue;  // warp-uniform
      const uint32_t key = has ? id[k] : 0u;
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
      const unsigned total = __reduce_add_sync(peers, has ? len[k] : 0u);
      int l3[3], h3[3];
      l3[0] = int(__reduce_min_sync(peers, unsigned(x + k)));
      h3[0] = int(__reduce_max_sync(peers, unsigned(x + k + int(len[k]) - 1)));
      if (one_row) {
        l3[1] = h3[1] = y;
        l3[2] = h3[2] = z;
      } else {
        l3[1] = int(__reduce_min_sync(peers, unsigned(y)));
        h3[1] = int(__reduce_max_sync(peers, unsigned(y)));
        l3[2] = int(__reduce_min_sync(peers, unsigned(z)));
        h3[2] = int(__reduce_max_sync(peers, unsigned(z)));
      }
      if (!has || lane != __ffs(peers) - 1) continue;
      const int slot = table_slot(keys, key);
      if (slot < 0) {
        box_update(lo + 3 * (long long)key, hi + 3 * (long long)key, counts + key, l3, h3, total);
        continue;
      }
      atomicAdd(cnt + slot, total);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        atomicMin(&slo[slot][a], l3[a]);
        atomicMax(&shi[slot][a], h3[a]);
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kSlots; t += blockDim.x) {
    const uint32_t id = keys[t];
    if (id) box_update(lo + 3 * (long long)id, hi + 3 * (long long)id, counts + id, slo[t], shi[t], cnt[t]);
  }
}

void launch_analyze(Context &ctx, const uint32_t *ids, Dims d, int *lo, int *hi, unsigned long long *counts) {
  if (d.n() <= 0) return;
  if (reinterpret_cast<uintptr_t>(ids) % 16 == 0 && d.sx % 4 == 0) {
    analyze4_kernel<<<blocks_for(d.n(), kQuadChunk), 256, 0, ctx.stream()>>>(ids, d, lo, hi, counts);
  } else {
    analyze_kernel<<<blocks_for(d.n(), kChunk), 256, 0, ctx.stream()>>>(ids, d, lo, hi, counts);
  }
  ++ctx.launches;
}

void launch_segmax(Context &ctx, const float *field, const uint32_t *ids, long long n, unsigned *best) {
  if (n <= 0) return;
  if (reinterpret_cast<uintptr_t>(field) % 16 == 0 && reinterpret_cast<uintptr_t>(ids) % 16 == 0) {
    segmax4_kernel<<<blocks_for(n, kQuadChunk), 256, 0, ctx.stream()>>>(field, ids, n, best);
  } else {
    segmax_kernel<<<blocks_for(n, kChunk), 256, 0, ctx.stream()>>>(field, ids, n, best);
  }
  ++ctx.launches;
}

__global__ void zero_to_inf_kernel(const uint32_t *__restrict__ ids, float *__restrict__ f, long long n,
                                   unsigned long long *count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool hit = i < n && ids[i] != 0 && f[i] == 0.0f;
  if (hit) f[i] = __uint_as_float(BK_INF_BITS);
  const unsigned many = __popc(__ballot_sync(0xFFFFFFFFu, hit));
  if (many && (threadIdx.x & 31) == 0) atomicAdd(count, (unsigned long long)many);
}

__global__ void fill_kernel(float *p, long long n, float v) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

struct FaceDesc {
  long long offset;
  int sx, sy, sz, a, b, c, fixed;
};

// grid (ceil(W * H / 256), faces): pixel (pb, pa) of slice f
__global__ void faces_kernel(const uint32_t *__restrict__ ids, const FaceDesc *faces, int W, int H, uint32_t *stack) {
  const FaceDesc f = faces[blockIdx.y];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)W * H) return;
  const int pb = int(i % W), pa = int(i / W);
  const int shape[3] = {f.sx, f.sy, f.sz};
  uint32_t v = 0;
  if (pa < shape[f.a] && pb < shape[f.b]) {
    int p[3];
    p[f.a] = pa;
    p[f.b] = pb;
    p[f.c] = f.fixed;
    v = ids[f.offset + p[0] + (long long)f.sx * (p[1] + (long long)f.sy * p[2])];
  }
  stack[i + (long long)W * H * blockIdx.y] = v;
}

// Per face component (ids of a face stack): pixel count, sums of the face coordinates pa and pb,
// the largest positive distance (float bits) and the first pixel (pa + fx * pb) with one.
__global__ void face_stats_kernel(const uint32_t *__restrict__ sids, const float *__restrict__ sdist,
                                  const FaceDesc *faces, int W, int H, unsigned long long *count,
                                  unsigned long long *sum_a, unsigned long long *sum_b, unsigned *max_bits,
                                  unsigned long long *first) {
  const FaceDesc f = faces[blockIdx.y];
  const int shape[3] = {f.sx, f.sy, f.sz};
  const int fx = shape[f.a], fy = shape[f.b];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)fx * fy) return;
  const int pb = int(i % fy), pa = int(i / fy);
  const long long src = pb + (long long)W * (pa + (long long)H * blockIdx.y);
  const uint32_t l = sids[src];
  if (!l) return;
  atomicAdd(count + l, 1ull);
  atomicAdd(sum_a + l, (unsigned long long)pa);
  atomicAdd(sum_b + l, (unsigned long long)pb);
  const float d = sdist[src];
  if (d > 0.0f) {
    atomicMax(max_bits + l, __float_as_uint(d));
    atomicMin(first + l, (unsigned long long)(pa + (long long)fx * pb));
  }
}

// The pixels at their component's largest positive distance: (component, pa, pb) triples.
__global__ void face_candidates_kernel(const uint32_t *__restrict__ sids, const float *__restrict__ sdist,
                                       const FaceDesc *faces, int W, int H, const unsigned *max_bits, int *n,
                                       int *out, long long capacity) {
  const FaceDesc f = faces[blockIdx.y];
  const int shape[3] = {f.sx, f.sy, f.sz};
  const int fx = shape[f.a], fy = shape[f.b];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)fx * fy) return;
  const int pb = int(i % fy), pa = int(i / fy);
  const long long src = pb + (long long)W * (pa + (long long)H * blockIdx.y);
  const uint32_t l = sids[src];
  if (!l) return;
  const float d = sdist[src];
  if (!(d > 0.0f) || __float_as_uint(d) != max_bits[l]) return;
  const int slot = atomicAdd(n, 1);
  if (slot < capacity) { out[3LL * slot] = int(l); out[3LL * slot + 1] = pa; out[3LL * slot + 2] = pb; }
}

Buffer<FaceDesc> face_descs(Context &ctx, const std::vector<Face> &faces) {
  std::vector<FaceDesc> h;
  for (const auto &f : faces) h.push_back({f.offset, f.d.sx, f.d.sy, f.d.sz, f.a, f.b, f.c, f.fixed});
  return to_device(ctx, h);
}

}  // namespace

std::vector<Box> analyze(Context &ctx, const uint32_t *ids, VolumeDims vd, int64_t count) {
  const Dims d{vd.sx, vd.sy, vd.sz};
  std::vector<int> lo(3 * (count + 1), INT32_MAX), hi(3 * (count + 1), -1);
  Buffer<int> dlo = to_device(ctx, lo), dhi = to_device(ctx, hi);
  Buffer<unsigned long long> counts(ctx, count + 1);
  counts.zero();
  launch_analyze(ctx, ids, d, dlo.data(), dhi.data(), counts.data());
  BK_CUDA(cudaGetLastError());
  lo = dlo.download();
  hi = dhi.download();
  auto c = counts.download();
  std::vector<Box> boxes(count + 1);
  for (int64_t id = 0; id <= count; ++id) {
    for (int a = 0; a < 3; ++a) { boxes[id].lo[a] = lo[3 * id + a]; boxes[id].hi[a] = hi[3 * id + a]; }
    boxes[id].count = (int64_t)c[id];
  }
  return boxes;
}

void neighbour_mask(Context &ctx, const uint32_t *ids, VolumeDims vd, uint32_t *out) {
  if (vd.n() <= 0) return;
  const dim3 grid((vd.sx + kMaskX - 1) / kMaskX, (vd.sy + kMaskY - 1) / kMaskY, (vd.sz + kMaskZ - 1) / kMaskZ);
  if (grid.y > 65535 || grid.z > 65535) throw std::invalid_argument("volume too large for the neighbour mask");
  const Dims d{vd.sx, vd.sy, vd.sz};
  if (reinterpret_cast<uintptr_t>(ids) % 16 == 0 && vd.sx % 4 == 0)
    mask_kernel<true><<<grid, dim3(kMaskX, kMaskY), 0, ctx.stream()>>>(ids, d, out);
  else
    mask_kernel<false><<<grid, dim3(kMaskX, kMaskY), 0, ctx.stream()>>>(ids, d, out);
  ++ctx.launches;
  BK_CUDA(cudaGetLastError());
}

std::vector<std::vector<Box>> analyze(Context &ctx, const uint32_t *ids, const std::vector<IdVolume> &volumes) {
  std::vector<long long> base(volumes.size() + 1, 0);
  for (size_t v = 0; v < volumes.size(); ++v) base[v + 1] = base[v] + volumes[v].count + 1;
  const long long total = base.back();
  cudaStream_t s = ctx.stream();
  Buffer<int> dlo(ctx, 3 * total), dhi(ctx, 3 * total);
  Buffer<unsigned long long> counts(ctx, total);
  dlo.fill_bytes(0x7F);  // 0x7F7F7F7F: above every coordinate
  dhi.fill_bytes(0xFF);  // -1
  counts.zero();
  for (size_t v = 0; v < volumes.size(); ++v) {
    const auto &iv = volumes[v];
    if (!iv.d.n() || !iv.count) continue;
    launch_analyze(ctx, ids + iv.offset, Dims{iv.d.sx, iv.d.sy, iv.d.sz}, dlo.data() + 3 * base[v],
                   dhi.data() + 3 * base[v], counts.data() + base[v]);
  }
  BK_CUDA(cudaGetLastError());
  std::vector<int> lo(3 * total), hi(3 * total);
  std::vector<unsigned long long> c(total);
  BK_CUDA(cudaMemcpyAsync(lo.data(), dlo.data(), lo.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
  BK_CUDA(cudaMemcpyAsync(hi.data(), dhi.data(), hi.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
  BK_CUDA(cudaMemcpyAsync(c.data(), counts.data(), c.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  ctx.synchronize();
  std::vector<std::vector<Box>> out(volumes.size());
  for (size_t v = 0; v < volumes.size(); ++v) {
    out[v].resize(volumes[v].count + 1);
    for (int64_t id = 0; id <= volumes[v].count; ++id) {
      const long long g = base[v] + id;
      for (int a = 0; a < 3; ++a) { out[v][id].lo[a] = lo[3 * g + a]; out[v][id].hi[a] = hi[3 * g + a]; }
      out[v][id].count = (int64_t)c[g];
    }
  }
  return out;
}

std::vector<std::vector<float>> segment_max(Context &ctx, const float *field, const uint32_t *ids,
                                            const std::vector<IdVolume> &volumes) {
  std::vector<long long> base(volumes.size() + 1, 0);
  for (size_t v = 0; v < volumes.size(); ++v) base[v + 1] = base[v] + volumes[v].count + 1;
  Buffer<unsigned> best(ctx, base.back());
  best.zero();
  for (size_t v = 0; v < volumes.size(); ++v) {
    const auto &iv = volumes[v];
    if (!iv.d.n() || !iv.count) continue;
    launch_segmax(ctx, field + iv.offset, ids + iv.offset, iv.d.n(), best.data() + base[v]);
  }
  BK_CUDA(cudaGetLastError());
  auto bits = best.download();
  std::vector<std::vector<float>> out(volumes.size());
  for (size_t v = 0; v < volumes.size(); ++v) {
    out[v].resize(volumes[v].count + 1);
    std::memcpy(out[v].data(), bits.data() + base[v], out[v].size() * sizeof(float));
  }
  return out;
}

std::vector<float> segment_max(Context &ctx, const float *field, const uint32_t *ids, long long n, int64_t count) {
  Buffer<unsigned> best(ctx, count + 1);
  best.zero();
  launch_segmax(ctx, field, ids, n, best.data());
  BK_CUDA(cudaGetLastError());
  auto bits = best.download();
  std::vector<float> out(count + 1);
  std::memcpy(out.data(), bits.data(), bits.size() * sizeof(float));
  return out;
}

long long zero_distances_to_infinity(Context &ctx, const uint32_t *ids, float *dbf, long long n) {
  if (n <= 0) return 0;
  Buffer<unsigned long long> count(ctx, 1);
  count.zero();
  zero_to_inf_kernel<<<blocks_for(n), 256, 0, ctx.stream()>>>(ids, dbf, n, count.data()); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  return (long long)count.download(1)[0];
}

void fill_float(Context &ctx, float *p, long long n, float value) {
  if (n <= 0) return;
  fill_kernel<<<blocks_for(n), 256, 0, ctx.stream()>>>(p, n, value); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
}

void extract_faces(Context &ctx, const uint32_t *ids, const std::vector<Face> &faces, int W, int H, uint32_t *stack) {
  if (faces.empty()) return;
  Buffer<FaceDesc> desc = face_descs(ctx, faces);
  faces_kernel<<<dim3(blocks_for((long long)W * H), unsigned(faces.size())), 256, 0, ctx.stream()>>>(
      ids, desc.data(), W, H, stack); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
}

FaceStats face_stats(Context &ctx, const uint32_t *stack_ids, const float *stack_dist, const std::vector<Face> &faces,
                     int W, int H, int64_t components) {
  FaceStats out;
  if (faces.empty()) return out;
  cudaStream_t s = ctx.stream();
  Buffer<FaceDesc> desc = face_descs(ctx, faces);
  const size_t k = size_t(components) + 1;
  Buffer<unsigned long long> count(ctx, k), sum_a(ctx, k), sum_b(ctx, k), first(ctx, k);
  Buffer<unsigned> max_bits(ctx, k);
  count.zero(); sum_a.zero(); sum_b.zero(); max_bits.zero();
  first.fill_bytes(0xFF);
  long long most = 0, pixels = 0;
  for (const auto &f : faces) {
    most = std::max(most, (long long)f.fx() * f.fy());
    pixels += (long long)f.fx() * f.fy();
  }
  const dim3 grid(blocks_for(most), unsigned(faces.size()));
  face_stats_kernel<<<grid, 256, 0, s>>>(stack_ids, stack_dist, desc.data(), W, H, count.data(), sum_a.data(),
                                         sum_b.data(), max_bits.data(), first.data()); ++ctx.launches;
  Buffer<int> n(ctx, 1), cand(ctx, 3 * std::max(pixels, 1LL));
  n.zero();
  face_candidates_kernel<<<grid, 256, 0, s>>>(stack_ids, stack_dist, desc.data(), W, H, max_bits.data(), n.data(),
                                              cand.data(), pixels); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  out.count = count.download();
  out.sum_a = sum_a.download();
  out.sum_b = sum_b.download();
  out.first = first.download();
  out.max_bits = max_bits.download();
  const int got = n.download(1)[0];
  out.candidates = cand.download(3 * size_t(std::min<long long>(got, pixels)));
  return out;
}

}  // namespace bk
