#pragma once
#include <cstdint>
#include <vector>

#include "runtime.hpp"

namespace bk {
// A volume's range [begin, end) of the arena, and where its id -> object table starts.
struct ArenaVolume {
  long long begin, end;
  int id_base;
};
// Voxels of every object over all volumes of the arena in one selection and one sort: grouped by
// global object index (object_of[id_base + id] >= 0), ascending in arena flat index. The picked
// voxels are also marked in `alive` (zeroed by the caller). `total` is the objects' voxel count.
Buffer<int> arena_object_voxels(Context &ctx, const uint32_t *ids, long long n, const std::vector<ArenaVolume> &volumes,
                                const std::vector<int> &object_of, int nobj, long long total, uint8_t *alive);
// Per object (voxels [begin[o], begin[o+1]) of the list, the last to `total`): its voxels by
// descending DAF (inf -> 0), ties -> higher flat first. `largest` is the largest object's voxel
// count; `wide` forces the (32, 64)-bit key even where 64 bits would hold it.
// In two steps: plan_target_orders makes every buffer (no stream work), run_target_orders only
// launches, so that a stream capture of it holds kernels and no allocations.
struct OrderPlan {
  Buffer<int> order;                        // the result
  Buffer<unsigned char> keys, sorted, scratch;
  size_t temp = 0;
  long long total = 0;
  int nobj = 0, lbits = 0, end_bit = 0;
  bool wide = false;
};
OrderPlan plan_target_orders(Context &ctx, long long total, int nobj, long long largest, bool wide = false);
void run_target_orders(Context &ctx, OrderPlan &plan, const int *vox, const float *daf, const int *begin);
Buffer<int> target_orders(Context &ctx, const int *vox, const float *daf, long long total, const int *begin, int nobj,
                          long long largest, bool wide = false);
}  // namespace bk
