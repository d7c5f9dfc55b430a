// Skeletonization of one or several label volumes (the reference's skeletonize / skeletonize_batch,
// skeletonize.cu:184-198 and batch.cu:430-515 of giorgioangel/brook).
#pragma once
#include <array>
#include <cstdint>
#include <memory>
#include <optional>
#include <vector>

#include "kernels.hpp"

namespace bk {

// TEASAR parameters; keys a caller leaves out take kimimaro.trace's defaults (skeleton.hpp:23-27).
struct Teasar {
  double scale = 10, constant = 10, pdrf_scale = 5000, pdrf_exponent = 16;
  double soma_detection = 1100, soma_acceptance = 4000, soma_scale = 0.5, soma_constant = 0;
  std::optional<int64_t> max_paths;
};

struct Options {
  Teasar teasar;
  std::array<float, 3> anisotropy{1, 1, 1};
  double dust = 1000;
  bool fix_branching = true, fix_borders = true;
  bool fill_holes = false;  // every component's voids filled before the EDT (BROOK_FILL_HOLES)
  bool fix_avocados = false;  // pits merged into the objects around them after the EDT (BROOK_FIX_AVOCADOS)
  std::optional<std::vector<int64_t>> object_ids;
  // extra targets per volume of the call (x, y, z in that volume's frame); volumes beyond the
  // vectors' ends have none
  std::vector<std::vector<Point>> targets_before, targets_after;
  bool device_output = false;  // keep vertices, edges and radii on the device (BROOK_DEVICE_OUTPUT)
};

// Packed skeletons of one volume: skeleton k has label labels[k], vertices
// [vertex_offsets[k], vertex_offsets[k+1]) (x, y, z physical, row major), the same range of
// radii, and edges [edge_offsets[k], edge_offsets[k+1]) local to the skeleton.
// With device output the three arrays live in `device_*` (same layouts; storage that outlives the
// context) and the host vectors stay empty.
struct Packed {
  std::vector<int64_t> labels, vertex_offsets{0}, edge_offsets{0};
  std::vector<float> vertices, radii;
  std::vector<uint32_t> edges;
  std::array<float, 3> anisotropy{1, 1, 1};
  std::shared_ptr<DeviceStorage> device_vertices, device_edges, device_radii;
  bool on_device() const { return device_vertices != nullptr; }
};

// A label volume already on the device, Fortran-ordered (x fastest), borrowed for the call.
struct DeviceVolume {
  const void *data = nullptr;
  int dtype = U32;
  VolumeDims d;
  const Slabs *slabs = nullptr;  // non-null: still arriving by slabs (kernels.hpp)
  // A crop of a larger volume (the out-of-core path): the EDT's walls per face (EdtVolume::faces;
  // -1: the black-border rule), the crop's corner in the larger volume (output vertices come out
  // in that volume's frame), and, when non-null, the border targets per component id (this
  // volume's frame) to use instead of the ones of this volume's own faces.
  int faces = -1;
  std::array<int, 3> origin{0, 0, 0};
  const std::vector<std::vector<Point>> *borders = nullptr;
};

std::vector<Packed> skeletonize(Context &ctx, const std::vector<DeviceVolume> &volumes, const Options &options);

// The volume's labels with every label not in `ids` set to 0 (same element type, on the device).
Buffer<unsigned char> select_labels(Context &ctx, const DeviceVolume &v, const std::vector<int64_t> &ids);

}  // namespace bk
