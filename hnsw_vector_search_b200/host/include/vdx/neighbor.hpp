#pragma once

// Result type and ranking shared by every index and by the GPU kernels.
// Mirrors include/vecdex/neighbor.hpp:10-25 of the reference: the order has to be identical for
// the GPU results to equal the reference's, so the definition is alike by necessity.

#include <cstdint>

namespace vdx {

// A stored vector's id: its insertion position, 0 .. size() - 1. 32 bits, as in the reference.
using Id = std::uint32_t;

// One search result: the distance under the index's metric (smaller is closer) and the id.
struct Neighbor {
    float distance;
    Id id;

    friend bool operator==(const Neighbor&, const Neighbor&) = default;
};

// Smaller distance first; equal distances by smaller id. A strict total order as long as no
// distance is NaN, which the indexes guarantee by rejecting non-finite input.
constexpr bool closer(const Neighbor& a, const Neighbor& b) noexcept {
    return a.distance < b.distance || (a.distance == b.distance && a.id < b.id);
}

}  // namespace vdx
