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

// The same contract with the table read as 4-slot buckets (16 bytes, one shared-memory load):
// an id lives in the first bucket of its sequence that had an empty slot when it was inserted,
// and slots only fill, so a lookup that meets a bucket with an empty slot and without the id
// knows the id is new. Most lookups read one bucket, where slot-by-slot linear probing walked
// the table's clusters one atomic at a time. A lane that loses a slot to another lane's CAS
// reads the bucket again; a lane that meets kProbes / 4 full buckets reports "unvisited".
__device__ __forceinline__ bool first_visit_bucket(std::uint32_t* table, std::uint32_t mask,
                                                   std::uint32_t id) {
    std::uint32_t b = (id * 2654435761u) & mask & ~3u;
    int full = 0;
#pragma unroll 1
    for (int step = 0; step < 2 * kProbes; ++step) {
        const uint4 s = *reinterpret_cast<const uint4*>(table + b);
        if (s.x == id || s.y == id || s.z == id || s.w == id) {
            return false;
        }
        const std::uint32_t e = s.x == kNoId ? 0u : s.y == kNoId ? 1u : s.z == kNoId ? 2u
                                : s.w == kNoId ? 3u : 4u;
        if (e < 4) {
            const std::uint32_t old = atomicCAS(table + b + e, kNoId, id);
            if (old == kNoId) {
                return true;
            }
            if (old == id) {
                return false;
            }
            continue;  // another lane took the slot: read the bucket again
        }
        if (++full >= kProbes / 4) {
            return true;
        }
        b = (b + 4) & mask;
    }
    return true;
}

// Copies `count` rows (ids in `ids`, shared) of `row_bytes` each from `base` into `dst`
// (shared, rows `dst_stride` bytes apart), 16 bytes per lane per step, and commits them as one
// cp.async group. `shift` is log2(row_bytes / 16) when that is a power of two up to 32 (several
// rows per warp-wide step, no division), else -1. kL1: copy through L1 (see cp_async16).
template <bool kL1 = false>
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
                cp_async16<kL1>(dst + r * dst_stride + (c << 4),
                                base + static_cast<std::size_t>(ids[r]) * row_bytes + (c << 4));
            }
        }
    } else {
        for (std::uint32_t r = 0; r < count; ++r) {
            const unsigned char* src = base + static_cast<std::size_t>(ids[r]) * row_bytes;
            for (std::uint32_t c = static_cast<std::uint32_t>(lane); c < chunks; c += 32) {
                cp_async16<kL1>(dst + r * dst_stride + (c << 4), src + (c << 4));
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

// R held in registers, for result capacities up to 64: lane l holds entries l and 32 + l
// (distance, id with the expanded bit); entries at r and beyond hold (+inf, kNoId). The
// shared-memory arrays (rd, rid) stay an exact mirror of R[0, r) — every write goes to both —
// so code after the walk reads R there; the walk itself reads the registers.
constexpr std::uint32_t kRegBeamCap = 64;

struct RegBeam {
    float d0, d1;
    std::uint32_t i0, i1;
};

__device__ __forceinline__ void reg_beam_init(RegBeam& b, float d, std::uint32_t id, int lane) {
    b.d0 = lane == 0 ? d : INFINITY;
    b.i0 = lane == 0 ? id : kNoId;
    b.d1 = INFINITY;
    b.i1 = kNoId;
}

// R[p] for a warp-uniform p.
__device__ __forceinline__ float reg_d(const RegBeam& b, int p) {
    return __shfl_sync(kFull, p < 32 ? b.d0 : b.d1, p & 31);
}
__device__ __forceinline__ std::uint32_t reg_id(const RegBeam& b, int p) {
    return __shfl_sync(kFull, p < 32 ? b.i0 : b.i1, p & 31);
}

__device__ __forceinline__ void reg_mark_expanded(RegBeam& b, int p, int lane) {
    if (lane == (p & 31)) {
        if (p < 32) {
            b.i0 |= kExpanded;
        } else {
            b.i1 |= kExpanded;
        }
    }
}

// first_unexpanded over the registers.
__device__ __forceinline__ int reg_first_unexpanded(const RegBeam& b, int from, int r, int lane) {
    const std::uint32_t m0 = __ballot_sync(kFull, lane >= from && lane < r && (b.i0 & kExpanded) == 0);
    if (m0 != 0) {
        return __ffs(m0) - 1;
    }
    const int l1 = 32 + lane;
    const std::uint32_t m1 = __ballot_sync(kFull, l1 >= from && l1 < r && (b.i1 & kExpanded) == 0);
    return m1 != 0 ? 32 + __ffs(m1) - 1 : r;
}

// merge_round (common.cuh) over the registers, with the same result: the full-list admission
// test, each candidate's position `lo` (the number of entries closer than it), the duplicate
// test (its id already in R), the rank among admitted candidates, entries at index i moved up by
// the number of admitted positions <= i, and everything at ef or beyond dropped. The candidates
// that pass the admission test are taken one at a time, broadcast to the warp: every lane
// compares them with its two entries, and two ballots count `lo` — no binary search, so a round
// costs a few shuffles and votes per surviving candidate (in a full list usually two or three
// of the ~13 scored). The new R is scattered into the shared-memory mirror (rd, rid) and read
// back into the registers. Returns the lowest position a candidate was kept at (0x7FFFFFFF if
// none).
template <typename Count>
__device__ __forceinline__ int reg_merge_round(RegBeam& b, float* rd, std::uint32_t* rid, int& r,
                                               int ef, float my_d, std::uint32_t my_id, bool valid,
                                               int lane, Count& dups) {
    if (r >= ef) {
        const float wd = reg_d(b, r - 1);
        const std::uint32_t wi = reg_id(b, r - 1) & kIdMask;
        valid = valid && closer(my_d, my_id, wd, wi);
    }
    const std::uint32_t vm = __ballot_sync(kFull, valid);
    if (vm == 0) {
        return 0x7FFFFFFF;
    }
    // Entries at r and beyond hold (+inf, kNoId): never closer than a candidate, never equal.
    const std::uint32_t e0 = b.i0 & kIdMask;
    const std::uint32_t e1 = b.i1 & kIdMask;
    const bool live0 = lane < r;
    const bool live1 = 32 + lane < r;
    std::uint32_t am = 0;
    int rank = 0;
    int s0 = 0;
    int s1 = 0;
    int lo = 0;
    for (std::uint32_t m = vm; m != 0; m &= m - 1) {
        const int j = __ffs(m) - 1;
        const float dj = __shfl_sync(kFull, my_d, j);
        const std::uint32_t ij = __shfl_sync(kFull, my_id, j);
        const bool dup = __any_sync(kFull, (live0 && e0 == ij) || (live1 && e1 == ij));
        if (!dup) {
            const int lj = __popc(__ballot_sync(kFull, live0 && closer(b.d0, e0, dj, ij))) +
                           __popc(__ballot_sync(kFull, live1 && closer(b.d1, e1, dj, ij)));
            am |= 1u << j;
            rank += closer(dj, ij, my_d, my_id) ? 1 : 0;
            s0 += lj <= lane ? 1 : 0;
            s1 += lj <= 32 + lane ? 1 : 0;
            lo = lane == j ? lj : lo;
        }
    }
    if (lane == 0) {
        dups += __popc(vm & ~am);
    }
    if (am == 0) {
        return 0x7FFFFFFF;
    }
    const bool adm = ((am >> lane) & 1u) != 0;
    const int p0 = lane + s0;
    const int p1 = 32 + lane + s1;
    const int newpos = lo + rank;
    const bool keep = adm && newpos < ef;
    if (live0 && p0 < ef) {
        rd[p0] = b.d0;
        rid[p0] = b.i0;
    }
    if (live1 && p1 < ef) {
        rd[p1] = b.d1;
        rid[p1] = b.i1;
    }
    if (keep) {
        rd[newpos] = my_d;
        rid[newpos] = my_id;
    }
    r = min(ef, r + __popc(am));
    __syncwarp();
    b.d0 = lane < r ? rd[lane] : INFINITY;
    b.i0 = lane < r ? rid[lane] : kNoId;
    b.d1 = 32 + lane < r ? rd[32 + lane] : INFINITY;
    b.i1 = 32 + lane < r ? rid[32 + lane] : kNoId;
    const int low = static_cast<int>(
        __reduce_min_sync(kFull, keep ? static_cast<std::uint32_t>(newpos) : 0x7FFFFFFFu));
    __syncwarp();
    return low;
}

}  // namespace vdx::dev
