#pragma once

// Recall measures, the reference's definitions (include/vecdex/recall.hpp:15-30).

#include <cstddef>
#include <cstdint>
#include <span>

#include "vdx/neighbor.hpp"

namespace vdx {

// |first k of found ∩ first k of truth| / k; a duplicate found id counts once.
double recall_at_k(std::span<const Neighbor> found, std::span<const std::int32_t> truth,
                   std::size_t k);

// Share of the first k found whose distance is at most the k-th true distance plus
// tolerance * max(|kth|, 1).
double threshold_recall_at_k(std::span<const Neighbor> found, float kth_true_distance,
                             std::size_t k, float tolerance = 1e-5F);

}  // namespace vdx
