// Shared device definitions of the brook_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace bk {

#define BK_INF_BITS 0x7f800000u
#define BK_UNCLAIMED 0xFFFFFFFFFFFFFFFFull

// 26-neighbour order shared by every kernel (the reference's tie rules are stated in it,
// common.cuh:33-47 of giorgioangel/brook): faces (-x,+x,-y,+y,-z,+z); the xy, yz and xz edges,
// each sign pair in lexicographic order; the corners lexicographic with z fastest.
// Bit k of a voxel's neighbour mask is neighbour k.
// (The lists as macros too, for kernels that want them as compile-time constants.)
#define BK_NEIGHBOUR_DX -1, 1, 0, 0, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, -1, -1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1
#define BK_NEIGHBOUR_DY 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, -1, -1, 1, 1, 0, 0, 0, 0, -1, -1, 1, 1, -1, -1, 1, 1
#define BK_NEIGHBOUR_DZ 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, 1
__constant__ int8_t c_dx[26] = {BK_NEIGHBOUR_DX};
__constant__ int8_t c_dy[26] = {BK_NEIGHBOUR_DY};
__constant__ int8_t c_dz[26] = {BK_NEIGHBOUR_DZ};
// neighbour k -> the index of the opposite offset
__constant__ int8_t c_opp[26] = {1, 0, 3, 2, 5, 4, 9, 8, 7, 6, 13, 12, 11, 10, 17, 16, 15, 14, 25, 24, 23, 22, 21, 20, 19, 18};
// dijkstra3d's neighbour order (its railroad joins the first rail in this order): the same faces
// and edges, corners (-,-,-)(+,-,-)(-,+,-)(-,-,+)(+,+,-)(+,-,+)(-,+,+)(+,+,+).
// rank: neighbour k -> position; inverse: position -> k.
__constant__ int8_t c_d3rank[26] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 21, 20, 24, 19, 23, 22, 25};
__constant__ int8_t c_d3inv[26] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 22, 20, 19, 24, 23, 21, 25};

struct Dims {
  int sx, sy, sz;
  __host__ __device__ long long n() const { return (long long)sx * sy * sz; }
};

__device__ __forceinline__ void unravel(int i, const Dims &d, int &x, int &y, int &z) {
  const int sxy = d.sx * d.sy;
  z = i / sxy;
  const int r = i - z * sxy;
  y = r / d.sx;
  x = r - y * d.sx;
}
// Flat offset of neighbour k (valid only when the neighbour is inside the volume).
__device__ __forceinline__ int nbr_offset(int k, const Dims &d) {
  return c_dx[k] + d.sx * (c_dy[k] + d.sy * c_dz[k]);
}

__device__ __forceinline__ uint32_t fbits(float f) { return __float_as_uint(f); }
__device__ __forceinline__ float bitsf(uint32_t b) { return __uint_as_float(b); }

// One vertex-weighted step: fl(d + f), advanced by one ulp where a positive f is absorbed, so that
// distances strictly increase along every step (the reference's brook_vw_step, common.cuh:113-127).
__device__ __forceinline__ float vw_step(float d, float f) {
  float c = __fadd_rn(d, f);
  if (c == d && f > 0.0f && d < __uint_as_float(BK_INF_BITS)) c = __uint_as_float(__float_as_uint(d) + 1u);
  return c;
}

// atomicMin on a non-negative float through its bit pattern (monotone as unsigned for f >= 0).
__device__ __forceinline__ float atomic_min_pos(float *addr, float value) {
  return __uint_as_float(atomicMin(reinterpret_cast<unsigned int *>(addr), __float_as_uint(value)));
}

// Loads that bypass L1: state that other threads of the block update with atomics.
template <class T> __device__ __forceinline__ T ld_cg(const T *p) { return __ldcg(p); }

// The penalty of one voxel (the reference's PDRF, batched_regular.inc:93-108 and its fused
// normalisation, trace_primitives.cu:119-129): a DBF of 0 counts as +inf and an infinite DAF as
// 0, then (1 - dbf * M) to the power 2^squarings by repeated squaring (squarings < 0: powf with
// `exponent`), times `scale`, plus daf * inv when inv is not 0; one rounding per operation.
__device__ __forceinline__ float pdrf_value(float dbf, float daf, float M, float inv, float scale, int squarings,
                                            float exponent) {
  if (dbf == 0.0f) dbf = __int_as_float(0x7f800000);
  float p = __fsub_rn(1.0f, __fmul_rn(dbf, M));
  if (squarings >= 0) for (int s = 0; s < squarings; ++s) p = __fmul_rn(p, p);
  else p = powf(p, exponent);
  p = __fmul_rn(p, scale);
  if (inv != 0.0f) {
    if (isinf(daf)) daf = 0.0f;
    p = __fadd_rn(p, __fmul_rn(daf, inv));
  }
  return p;
}

}  // namespace bk
