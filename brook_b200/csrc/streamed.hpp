// Out-of-core skeletonization of host volumes larger than the device's memory (streamed.cu).
#pragma once
#include <array>
#include <memory>
#include <vector>

#include "pipeline.hpp"

namespace bk {

// A label volume in host memory with byte strides per axis (x, y, z).
struct HostVolume {
  const void *data = nullptr;
  int dtype = U32;
  VolumeDims d;
  std::array<long long, 3> strides{0, 0, 0};
};

// A host array that is not initialised when made (a volume's worth of ids is written in full).
template <class T>
struct HostArray {
  std::unique_ptr<T[]> p;
  size_t n = 0;
  void resize(size_t count) {
    p.reset(count ? new T[count] : nullptr);
    n = count;
  }
  T *data() { return p.get(); }
  const T *data() const { return p.get(); }
  size_t size() const { return n; }
  T &operator[](size_t i) { return p[i]; }
  const T &operator[](size_t i) const { return p[i]; }
};

// The components of a host volume, computed slab by slab on the device: ids 1..count by ascending
// first flat index (the in-core numbering), per voxel in host memory.
struct StreamedComponents {
  VolumeDims d;
  int64_t count = 0;
  HostArray<uint32_t> ids;        // F order, 0 = background
  std::vector<int64_t> mapping;   // id -> original label (count + 1 entries)
  std::vector<int64_t> roots;     // id - 1 -> first flat index
  std::vector<Box> boxes;         // id -> box and voxel count (entry 0 unused)
  int slabs = 0;
};

// The device-memory budget of a streamed call: `requested` bytes as given (a slab still holds one
// plane and a batch one crop), or with 0 the environment's BROOK_STREAM_BUDGET_MB (a positive
// number of MiB), else a quarter of the device's free memory and at least 64 MiB.
size_t stream_budget(size_t requested);

StreamedComponents connected_components_streamed(Context &ctx, const HostVolume &labels, size_t budget,
                                                 const std::vector<int64_t> *object_ids);

// The multi-label EDT of a host volume (the in-core brook_edt's field, bit for bit) into `out` (host,
// n floats, Fortran order): components by slabs, then the x and y passes slab by slab and the z
// pass by tiles of whole columns, each piece staged through the device within the budget.
void edt_streamed(Context &ctx, const HostVolume &labels, const float aniso[3], bool black_border, size_t budget,
                  float *out);

// The skeletons skeletonize gives for the whole volume (same skeletons, same order), computed with
// a bounded device footprint: components from slabs, then every traced component in its bounding
// box as a crop (EDT walls where the box meets other voxels, the volume's border rule where it
// meets the volume's edge, border targets from the whole volume's faces), crops batched to the
// budget, and the crops' skeletons merged per label. fill_holes and fix_avocados are refused.
Packed skeletonize_streamed(Context &ctx, const HostVolume &labels, const Options &options, size_t budget);

}  // namespace bk
