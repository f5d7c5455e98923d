#pragma once

// Device building blocks of a best-first walk over one HNSW layer, shared by the search kernel
// (search.cu) and the graph builder (build.cu): the shared-memory visited filter, the row gather
// into shared memory, and the scan for R's first unexpanded entry.

#include <cstdint>

#include "common.cuh"

namespace vdx::dev {

constexpr int kProbes = 16;

// True if `id` was not seen before in this query's layer-0 search (inserts it). Never returns
// false for an unseen id.
__device__ __forceinline__ bool first_visit(std::uint32_t* table, std::uint32_t mask,
                                            std::uint32_t id) {
    std::uint32_t h = (id * 2654435761u) & mask;
#pragma unroll 1
    for (int p = 0; p < kProbes; ++p) {
        const std::uint32_t old = atomicCAS(table + h, kNoId, id);
        if (old == kNoId) {
            return true;
        }
        if (old == id) {
            return false;
        }
        h = (h + 1) & mask;
    }
    return true;
}

// Copies `count` rows (ids in `ids`, shared) of `row_bytes` each from `base` into `dst`
// (shared, rows `dst_stride` bytes apart), 16 bytes per lane per step, and commits them as one
// cp.async group. `shift` is log2(row_bytes / 16) when that is a power of two up to 32 (several
// rows per warp-wide step, no division), else -1.
__device__ __forceinline__ void gather_rows(unsigned char* dst, std::uint32_t dst_stride,
                                            const unsigned char* base, const std::uint32_t* ids,
                                            std::uint32_t count, std::uint32_t row_bytes, int shift,
                                            int lane) {
    const std::uint32_t chunks = row_bytes >> 4;
    if (shift >= 0) {
        const std::uint32_t per_step = 32u >> shift;
        const std::uint32_t r_in = static_cast<std::uint32_t>(lane) >> shift;
        const std::uint32_t c = static_cast<std::uint32_t>(lane) & (chunks - 1);
        for (std::uint32_t r0 = 0; r0 < count; r0 += per_step) {
            const std::uint32_t r = r0 + r_in;
            if (r < count) {
                cp_async16(dst + r * dst_stride + (c << 4),
                           base + static_cast<std::size_t>(ids[r]) * row_bytes + (c << 4));
            }
        }
    } else {
        for (std::uint32_t r = 0; r < count; ++r) {
            const unsigned char* src = base + static_cast<std::size_t>(ids[r]) * row_bytes;
            for (std::uint32_t c = static_cast<std::uint32_t>(lane); c < chunks; c += 32) {
                cp_async16(dst + r * dst_stride + (c << 4), src + (c << 4));
            }
        }
    }
    cp_async_commit();
}

__device__ __forceinline__ int chunk_shift(std::uint32_t row_bytes) {
    const std::uint32_t chunks = row_bytes >> 4;
    if (chunks == 0 || chunks > 32 || (chunks & (chunks - 1)) != 0) {
        return -1;
    }
    return __ffs(chunks) - 1;
}

// Index of the first unexpanded entry in R[from, r), or r if there is none.
__device__ __forceinline__ int first_unexpanded(const std::uint32_t* rid, int from, int r,
                                                int lane) {
    for (int base = from & ~31; base < r; base += 32) {
        const int i = base + lane;
        const bool open = i >= from && i < r && (rid[i] & kExpanded) == 0;
        const std::uint32_t m = __ballot_sync(kFull, open);
        if (m != 0) {
            return base + __ffs(m) - 1;
        }
    }
    return r;
}

}  // namespace vdx::dev
