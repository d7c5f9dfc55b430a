#pragma once
#include <cstdint>

#include "runtime.hpp"

namespace bk {
// Voxels of every object (rank[id] >= 0), grouped by object rank and ascending in flat index.
Buffer<int> object_voxels(Context &ctx, const uint32_t *ids, long long n, const int *rank, int nobj, long long total);
// Per object [begin, end): its voxels by descending DAF (inf -> 0), ties -> higher flat first.
Buffer<int> target_orders(Context &ctx, const int *vox, const float *daf, long long total, const int *begin,
                          const int *end, int nobj);
}  // namespace bk
