// Canonical post-processing of packed skeletons on the device (post.cu).
#pragma once
#include <memory>

#include "pipeline.hpp"

namespace bk {

// The steps of the reference's canonical post-processing (post.cu:646-650 of giorgioangel/brook):
// kPostprocess runs remove_dust(a), remove_loops, join_components, remove_ticks(b) and
// prune_unused in that order.
enum PostStep { kPostprocess = 0, kRemoveDust = 1, kRemoveLoops = 2, kJoinComponents = 3, kRemoveTicks = 4,
                kPruneUnused = 5 };

// One step (or the whole chain) on a packed set, host or device; the result is on the device.
Packed post_process(Context &ctx, const Packed &input, int step, double a, double b);

// The component id (the smallest global vertex id of its connected component) of every vertex, as
// int64 on the device; *count receives the vertex count.
std::shared_ptr<DeviceStorage> skeleton_components(Context &ctx, const Packed &input, size_t *count);

}  // namespace bk
