// Merge of skeleton fragments placed at physical origins (merge.cu).
#pragma once
#include <array>
#include <vector>

#include "pipeline.hpp"

namespace bk {

// One skeleton per label over all fragments (fragment f's vertices shifted by origins[f]); the
// result's arrays are on the device.
Packed merge_fragments(Context &ctx, const std::vector<const Packed *> &fragments,
                       const std::vector<std::array<float, 3>> &origins);

}  // namespace bk
