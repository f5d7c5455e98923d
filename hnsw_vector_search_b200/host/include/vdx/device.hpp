#pragma once

// The device mirror of an HNSW graph, as the search kernels read it from HBM.
//
//   vectors    n rows of the traversal copy (FP32, BF16, or FP8 E4M3 plus one FP32 scale at the
//              end of each row), each row padded to a multiple of 16 bytes so every row can be
//              gathered with 16-byte cp.async copies;
//   vectors32  the FP32 rows (the traversal copy itself in FP32 mode), used for exact re-ranking;
//   links0     n blocks of `stride0` u32 (2M rounded up to a multiple of 4): the node's layer-0
//              neighbors in link order, then 0xFFFFFFFF in every unused slot, so a block needs no
//              count and one block of M = 16 is exactly one 128-byte line;
//   upper_at   n u32: for a node with level >= 1, the index of its layer-1 block in links_up;
//   links_up   the upper-layer blocks, `stride_up` u32 each (M rounded up to 4), same sentinel
//              padding, in the file's node-then-layer order;
//   upper copy what the greedy descent reads, in one allocation kept resident in L2 by an
//              access-policy window on the descent launches: `upper_aug`, every upper block as
//              [the ids (stride_up u32) | each id's upper_at (stride_up u32)], and `upper_rows`,
//              the traversal row of every node with upper layers at the index of its first upper
//              block (row_bytes each). The descent then gathers from a few tens of MB instead of
//              from rows scattered over the whole vector array. Null when there are no upper
//              layers.
// Node ids on the device must stay below 2^31 (bit 31 marks expanded entries in the kernels'
// result lists); a B200 could not hold that many 4-byte-per-component vectors anyway.

#include <cstddef>
#include <cstdint>

namespace vdx {

struct DeviceGraphView {
    const void* vectors;
    const float* vectors32;
    const std::uint32_t* links0;
    const std::uint32_t* upper_at;
    const std::uint32_t* links_up;
    std::uint32_t n;
    std::uint32_t dim;
    std::uint32_t row_bytes;    // bytes per traversal row (16-byte multiple)
    std::uint32_t row32;        // floats per FP32 row (dim rounded up to 4)
    std::uint32_t stride0;      // u32 per layer-0 block
    std::uint32_t cap0;         // 2M
    std::uint32_t stride_up;    // u32 per upper block
    std::uint32_t cap_up;       // M
    std::uint32_t max_level;
    std::uint32_t entry;
    std::uint32_t metric;       // 0 L2, 1 inner product, 2 cosine
    std::uint32_t precision;    // 0 FP32, 1 BF16, 2 FP8
    const std::uint32_t* upper_aug = nullptr;       // see "upper copy" above (or null)
    const unsigned char* upper_rows = nullptr;
    std::uint32_t entry_ua = 0;                     // upper_at of the entry point
    const void* l2_window = nullptr;                // the upper copy's allocation
    std::size_t l2_window_bytes = 0;                // (within the device's window limit)
    float l2_hit_ratio = 0.0F;                      // share of the window the L2 set-aside holds
};

// Owns the device allocations behind a DeviceGraphView.
struct DeviceGraph {
    DeviceGraphView view{};
    int device = 0;
    void* vectors_alloc = nullptr;   // traversal copy when it is not the FP32 rows
    void* vectors32_alloc = nullptr;
    void* links0_alloc = nullptr;
    void* upper_at_alloc = nullptr;
    void* links_up_alloc = nullptr;
    void* upper_copy_alloc = nullptr;
    std::size_t bytes = 0;           // total device bytes held
    ~DeviceGraph();
};

}  // namespace vdx
