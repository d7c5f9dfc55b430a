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
// ids (per voxel: id 1..K, 0 = background). `planar`: 8-connected within each z-slice only.
ComponentsResult connected_components(Context &ctx, const void *labels, int dtype, VolumeDims d, uint32_t *ids,
                                      bool planar = false);
// The same for several volumes laid out back to back in one flat space (offsets in order, no
// gaps): ids + offset receives each volume's ids; one flatten, scan and download for all.
// Slabs of a volume still being copied to the device: z planes [previous end, end) are there once
// the event has completed (events in copy order, the last end is the volume's depth; each end but
// the last is a multiple of 8, the union tiles' depth).
using Slabs = std::vector<std::pair<int, cudaEvent_t>>;
struct CcVolume {
  const void *labels;
  int dtype;
  VolumeDims d;
  long long offset;
  const Slabs *slabs = nullptr;  // null: the labels are all there
};
std::vector<ComponentsResult> connected_components(Context &ctx, const std::vector<CcVolume> &volumes, uint32_t *ids,
                                                   bool planar = false);

// ---- EDT (edt.cu) ----
// Squared-then-rooted anisotropic distance of every voxel to the nearest voxel of a different id
// (the volume edge counts with black_border); background gets 0. dims = 2 skips the z pass: every
// z-slice is then an image of its own.
void edt(Context &ctx, const uint32_t *ids, VolumeDims d, const float aniso[3], bool black_border, int dims,
         float *out);

// The 3D EDT of several volumes of one flat index space (ids and out share the offsets): the x
// pass volume by volume, the y and z passes over every volume's lines in one launch each.
// The two halves of edt() for a volume taken in pieces (a host volume streamed through the
// device): the x and y passes of a stack of z-slices, leaving squared distances (not rooted), and
// the z pass of a block of whole columns over such squared distances, rooting them. Each line is
// computed as edt() computes it, so the pieces give edt()'s field.
void edt_xy_squared(Context &ctx, const uint32_t *ids, VolumeDims d, const float aniso[3], bool black_border, float *D);
void edt_z_finish(Context &ctx, const uint32_t *ids, VolumeDims d, float wz, bool black_border, float *D);
struct EdtVolume {
  long long offset;
  VolumeDims d;
  bool black_border;
  // Per-face walls (bit 2a: the low face of axis a, bit 2a + 1: its high face) for a crop of a
  // larger volume; -1: every face or none, by black_border.
  int faces = -1;
};
void edt_volumes(Context &ctx, const uint32_t *ids, const std::vector<EdtVolume> &volumes, const float aniso[3],
                 float *out);
// The black-border 2D EDT of a (W, H, groups * per_group) stack of images whose group g (per_group
// consecutive slices) has spacing wx[g] along x and wy[g] along y: what edt(..., dims = 2) gives each
// group, with the y passes of all groups in one launch.
void edt_planes(Context &ctx, const uint32_t *ids, int W, int H, int groups, int per_group, const float wx[3],
                const float wy[3], float *out);

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
// Several volumes of one flat index space (ids + offset, component ids 1..count each): one launch
// per volume, one download for all.
struct IdVolume {
  long long offset;
  VolumeDims d;
  int64_t count;
};
std::vector<std::vector<Box>> analyze(Context &ctx, const uint32_t *ids, const std::vector<IdVolume> &volumes);
// ---- hole filling (holes.cu) ----
// The components of each volume (ids + offset, boxes by id as analyze gives them) with their voids
// filled as the reference's fill_all_holes leaves them; returns the voxels filled. The ids change
// in place; the boxes are the ones before filling.
struct HoleVolume {
  long long offset;
  VolumeDims d;
  const std::vector<Box> *boxes;
};
long long fill_holes(Context &ctx, uint32_t *ids, const std::vector<HoleVolume> &volumes);
// The voids of a component in a box: the box's voxels that are not the id and not 6-connected,
// through such voxels, to a face of the box (fill_voids' rule). All boxes at once; returns per void
// voxel its flat index, its box and the id it holds, and per box the count.
struct VoidBox {
  long long vol_offset;
  VolumeDims d;
  Box box;
  uint32_t id;
};
struct Voids {
  std::vector<int> voxel, box;
  std::vector<uint32_t> held;
  std::vector<long long> count;
};
Voids component_voids(Context &ctx, const uint32_t *ids, const std::vector<VoidBox> &boxes);

// ---- the avocado stage (avocado.cpp) ----
// One volume's component ids (ids, device, 1..cc.count) and distance field (dbf, device) after the
// reference's fix_avocados: pits merged into the objects around them, ids renumbered by first voxel
// (cc's count, mapping and first voxels follow), the field refreshed by the EDT when a pass merged.
// Returns the passes run.
int fix_avocados(Context &ctx, uint32_t *ids, float *dbf, VolumeDims d, ComponentsResult &cc, double threshold,
                 const float aniso[3], bool black_border);
// A foreground voxel at distance zero (background the avocado stage painted without a refresh)
// becomes +inf: the tracer's penalty, invalidation reach and radius. Returns how many there were.
long long zero_distances_to_infinity(Context &ctx, const uint32_t *ids, float *dbf, long long n);
std::vector<std::vector<float>> segment_max(Context &ctx, const float *field, const uint32_t *ids,
                                            const std::vector<IdVolume> &volumes);
// 26-bit same-id neighbour mask of every voxel (0 for background).
void neighbour_mask(Context &ctx, const uint32_t *ids, VolumeDims d, uint32_t *out);
// Per id the largest value of `field` (non-negative, finite), as float bits.
std::vector<float> segment_max(Context &ctx, const float *field, const uint32_t *ids, long long n, int64_t count);
void fill_float(Context &ctx, float *p, long long n, float value);
// One face of a volume whose ids start at ids + offset: the pixels with p[c] = fixed, pixel (pa, pb)
// = (p[a], p[b]), fx = extent of a, fy = extent of b.
struct Face {
  long long offset;
  VolumeDims d;
  int a, b, c, fixed;
  int fx() const { return a == 0 ? d.sx : a == 1 ? d.sy : d.sz; }
  int fy() const { return b == 0 ? d.sx : b == 1 ? d.sy : d.sz; }
};
// Every face into its own z-slice of a (W, H, faces) stack: stack[pb + W * (pa + H * f)], zero
// beyond the face's (fy, fx) corner.
void extract_faces(Context &ctx, const uint32_t *ids, const std::vector<Face> &faces, int W, int H, uint32_t *stack);

// Per component of a face stack (entry 0 unused): pixel count, sums of pa and pb, the largest
// positive distance as float bits (0: none), the first pixel pa + fx * pb with a positive
// distance (all ones: none), and every pixel at its component's largest positive distance as
// (component, pa, pb) triples.
struct FaceStats {
  std::vector<unsigned long long> count, sum_a, sum_b, first;
  std::vector<unsigned> max_bits;
  std::vector<int> candidates;
};
FaceStats face_stats(Context &ctx, const uint32_t *stack_ids, const float *stack_dist, const std::vector<Face> &faces,
                     int W, int H, int64_t components);

// ---- border targets (borders.cpp) ----
using Point = std::array<int64_t, 3>;
// Per volume, per component id: its border targets in the order the reference visits them. All
// faces of all volumes run through one planar CCL and three planar EDTs.
struct BorderVolume {
  long long offset;  // where the volume's ids start
  VolumeDims d;
  int64_t count;     // component ids 1..count
};
// given_stack: the volumes' faces already in the layout extract_faces writes (a device array of
// W * H * faces, from face_list's order and extents), used instead of reading them from ids.
std::vector<std::vector<std::vector<Point>>> border_targets(Context &ctx, const uint32_t *ids,
                                                            const std::vector<BorderVolume> &volumes,
                                                            const float aniso[3], const uint32_t *given_stack = nullptr);
// The faces of the volumes in the border stage's stack order, and the stack's slice extents.
std::vector<Face> face_list(const std::vector<BorderVolume> &volumes, int &W, int &H);

}  // namespace bk
