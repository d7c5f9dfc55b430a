// Skeleton assembly on the device: the reference's assemble_paths (assembly.cu:88-174) with the
// consolidate semantics of skeleton.cpp:13-40.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

#include "runtime.hpp"

namespace bk {

// The paths that make skeletons (two or more vertices), in output order: skeleton `group[p]`
// takes path p's vertices store[src[p] .. src[p] + len[p]), flat indices into the arena of
// volume `volume[p]`. Groups are numbered in output order (volume-major).
struct AssemblyPaths {
  std::vector<int> src, len, group, volume;
  int groups = 0;
};

// Packed skeletons of every group: per skeleton its vertices (the unique path voxels sorted by
// (x, y, z), as physical coordinates), the radius at each (the DBF), and its edges (consecutive
// path vertices, (lower, higher) local index, sorted, unique); vertices on no edge are dropped.
struct AssemblyResult {
  Buffer<float> vertices;  // V x 3, row major
  Buffer<float> radii;     // V
  Buffer<uint32_t> edges;  // E x 2, row major, local to the skeleton
  std::vector<int64_t> vertex_offsets, edge_offsets;  // groups + 1 each
};

// Arena r starts at arena_offset[r] with shape arena_dims[r]; its voxel (x, y, z) is the output
// vertex (x, y, z) + arena_origin[r] (a soma's private crop lies at its box corner in its volume).
AssemblyResult assemble(Context &ctx, const int *store, const float *dbf, const AssemblyPaths &paths,
                        const std::vector<long long> &arena_offset, const std::vector<std::array<int, 3>> &arena_dims,
                        const std::vector<std::array<int, 3>> &arena_origin, const float anisotropy[3]);

}  // namespace bk
