// Host entry points of the brook_b200 kernels. Every volume is Fortran-ordered (x fastest) with
// flat index i = x + sx * (y + sy * z) below 2^31.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

#include "runtime.hpp"

namespace bk {

struct Dims;

enum LabelType { U8 = 0, U16 = 1, U32 = 2, U64 = 3, I8 = 4, I16 = 5, I32 = 6, I64 = 7 };
size_t label_bytes(int dtype);

struct VolumeDims {
  int sx = 0, sy = 0, sz = 0;
  long long n() const { return (long long)sx * sy * sz; }
};

// ---- connected components (ccl.cu) ----
struct ComponentsResult {
  int64_t count = 0;             // K
  std::vector<int64_t> mapping;  // id -> original label (entry 0 unused), K + 1 entries
  std::vector<int64_t> roots;    // id - 1 -> first flat index of the component
};
// 26-connected components of equal nonzero labels, ids by ascending first flat index, written to
// ids (per voxel: id 1..K, 0 = background).
ComponentsResult connected_components(Context &ctx, const void *labels, int dtype, VolumeDims d, uint32_t *ids);

// ---- EDT (edt.cu) ----
// Squared-then-rooted anisotropic distance of every voxel to the nearest voxel of a different id
// (the volume edge counts with black_border); background gets 0. dims = 2 skips the z pass.
void edt(Context &ctx, const uint32_t *ids, VolumeDims d, const float aniso[3], bool black_border, int dims,
         float *out);

// EDT of uint32 labels with no device allocation (a fixed file-scope scratch in edt.cu); see there.
void edt_fixed_scratch(const uint32_t *labels, VolumeDims d, const float aniso[3], bool black_border, float *out,
                       cudaStream_t stream);
size_t edt_fixed_scratch_bytes();

// ---- preamble (prep.cu) ----
struct Box {
  int lo[3], hi[3];
  int64_t count;
};
std::vector<Box> analyze(Context &ctx, const uint32_t *ids, VolumeDims d, int64_t count);
// 26-bit same-id neighbour mask of every voxel (0 for background).
void neighbour_mask(Context &ctx, const uint32_t *ids, VolumeDims d, uint32_t *out);
// Per id the largest value of `field` (non-negative, finite), as float bits.
std::vector<float> segment_max(Context &ctx, const float *field, const uint32_t *ids, long long n, int64_t count);
void fill_float(Context &ctx, float *p, long long n, float value);
// Extract one face of `ids` as a (fy, fx, 1) plane: plane[pb + fy * pa] = ids[p[a]=pa, p[b]=pb, p[c]=fixed].
void extract_face(Context &ctx, const uint32_t *ids, VolumeDims d, int a, int b, int c, int fixed, uint32_t *plane);

// ---- border targets (borders.cpp) ----
using Point = std::array<int64_t, 3>;
std::vector<std::vector<Point>> border_targets(Context &ctx, const uint32_t *ids, VolumeDims d, int64_t count,
                                               const float aniso[3]);

}  // namespace bk
