// Graph construction on the GPU: batched parallel insertion into the device mirror.
//
// The reference inserts one node at a time (src/hnsw.cpp:295-409): a greedy walk down to the
// node's level, then on each of its layers a best-first search with ef_construction for
// candidates, the neighbor-selection heuristic for M of them, the node's own links, and links
// back from each chosen neighbor (a full neighbor list is re-selected with the node added). Its
// parallel add runs these inserts concurrently, each seeing whatever the others have linked.
//
// Here a batch of nodes is inserted at once, each by one warp, in three kernels:
//   1. build_search_kernel  the walk and the per-layer candidate searches of every node of the
//                           batch, against the graph as it was before the batch;
//   2. build_select_kernel  the heuristic per (node, layer), the node's own lists, and one
//                           proposal per chosen neighbor into that neighbor's proposal slots;
//   3. build_link_kernel    per neighbor list with proposals: append them, or, if the list
//                           would overflow, re-select it from the old links plus the proposals.
// Nodes of one batch do not see each other (as concurrent inserts of the reference's parallel
// add may not), so batches stay small against the graph: a 32nd of its size, at most 8192.
// The first 1024 nodes are inserted one by one on the host, exactly as the serial build. Levels
// are drawn in the serial order before anything is linked, so the layer structure is the serial
// build's. A node that raises the top layer ends its batch and becomes the entry point.
//
// Every loop is bounded (walks by the node count, selections by the list sizes); no kernel waits
// on another thread. Distances are the reference's (`thread_distance`, `pair_distance`).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <format>
#include <numeric>
#include <stdexcept>
#include <vector>

#include "beam.cuh"
#include "common.cuh"
#include "gpu_runtime.cuh"
#include "vdx/device.hpp"
#include "vdx/hnsw.hpp"
#include "../host/src/internal.hpp"

namespace vdx::dev {
namespace {

constexpr std::uint32_t kProposals = 64;    // proposal slots per neighbor list per batch
constexpr std::uint32_t kSeedNodes = 1024;  // inserted one by one on the host first
constexpr std::uint32_t kMaxBatch = 8192;
constexpr int kBuildWarps = 4;              // warps per block of the search kernel

struct BuildArgs {
    DeviceGraphView g;                 // mutable through the owning allocations
    std::uint32_t* links0;
    std::uint32_t* links_up;
    const std::uint8_t* levels;        // [n]
    const std::uint32_t* up_owner;     // [upper blocks]: owning node
    std::uint32_t n_up;                // upper blocks
    std::uint32_t first, count;        // the batch: nodes [first, first + count)
    std::uint32_t entry, max_level;    // the graph before the batch
    std::uint32_t M, ef, efcap, hash_slots, rows_cap;
    const std::uint32_t* cand_at;      // [count]: candidate slot of the node's layer 0 (layer l at + l)
    std::uint32_t* cand_ids;           // [slots][efcap]
    float* cand_d;
    std::uint32_t* cand_n;             // [slots]
    std::uint32_t* prop_count;         // [n + n_up]
    std::uint32_t* prop_ids;           // [n + n_up][kProposals]
    float* prop_d;
    std::uint32_t* touched;            // [n + n_up]: lists that received proposals
    std::uint32_t* touched_n;
    std::uint32_t* claim;              // work counter of the search kernel
    // per-warp shared-memory layout
    std::uint32_t warp_bytes, off_r, off_hash, off_links, off_rows, off_fresh, off_ap;
};

__device__ __forceinline__ std::uint32_t* block_of(const BuildArgs& a, std::uint32_t node,
                                                   std::uint32_t layer) {
    return layer == 0 ? a.links0 + static_cast<std::size_t>(node) * a.g.stride0
                      : a.links_up + static_cast<std::size_t>(a.g.upper_at[node] + layer - 1) * a.g.stride_up;
}

// The proposal list of (node, layer): layer-0 lists are 0..n-1, upper lists n + block index.
__device__ __forceinline__ std::uint32_t list_of(const BuildArgs& a, std::uint32_t node,
                                                 std::uint32_t layer) {
    return layer == 0 ? node : a.g.n + a.g.upper_at[node] + layer - 1;
}

template <bool kL2>
__device__ __forceinline__ float vec_distance(const BuildArgs& a, std::uint32_t x, std::uint32_t y) {
    return thread_distance<kL2>(a.g.vectors32 + static_cast<std::size_t>(x) * a.g.row32,
                                a.g.vectors32 + static_cast<std::size_t>(y) * a.g.row32, a.g.dim);
}

// ---------------------------------------------------------------------------------------------
// 1. Candidate searches.

template <bool kL2>
__global__ void __launch_bounds__(kBuildWarps * 32) build_search_kernel(const BuildArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = static_cast<int>(threadIdx.x & 31);
    const int warp = static_cast<int>(threadIdx.x >> 5);
    unsigned char* ws = smem + static_cast<std::size_t>(warp) * a.warp_bytes;
    float* q = reinterpret_cast<float*>(ws);
    float* rd = reinterpret_cast<float*>(ws + a.off_r);
    std::uint32_t* rid = reinterpret_cast<std::uint32_t*>(ws + a.off_r + a.efcap * 4);
    std::uint32_t* table = reinterpret_cast<std::uint32_t*>(ws + a.off_hash);
    std::uint32_t* lbuf = reinterpret_cast<std::uint32_t*>(ws + a.off_links);
    unsigned char* rows = ws + a.off_rows;
    std::uint32_t* fresh = reinterpret_cast<std::uint32_t*>(ws + a.off_fresh);
    int* ap = reinterpret_cast<int*>(ws + a.off_ap);
    const DeviceGraphView& g = a.g;
    const auto* vecs = reinterpret_cast<const unsigned char*>(g.vectors32);
    const std::uint32_t row_bytes = g.row32 * 4;
    const std::uint32_t stride_s = padded_row_stride(row_bytes);
    const int shift = chunk_shift(row_bytes);
    const int rounds_cap = static_cast<int>(a.rows_cap < 16 ? a.rows_cap : 16);
    const unsigned char* const my_row =
        rows + static_cast<std::uint32_t>(min(lane & 15, rounds_cap - 1)) * stride_s;
    const int half = lane >> 4;
    const std::uint32_t hmask = a.hash_slots - 1;

    for (;;) {
        std::uint32_t i = 0;
        if (lane == 0) {
            i = atomicAdd(a.claim, 1u);
        }
        i = __shfl_sync(kFull, i, 0);
        if (i >= a.count) {
            break;
        }
        const std::uint32_t v = a.first + i;
        const std::uint32_t level = a.levels[v];
        const std::uint32_t top = level < a.max_level ? level : a.max_level;
        for (std::uint32_t e = lane; e < g.row32; e += 32) {
            q[e] = g.vectors32[static_cast<std::size_t>(v) * g.row32 + e];
        }
        __syncwarp();

        // Scores up to rounds_cap rows listed in fresh[s0, s0 + cnt); lane < cnt gets row lane.
        const auto score = [&](int s0, int cnt) {
            gather_rows(rows, stride_s, vecs, fresh + s0, static_cast<std::uint32_t>(cnt), row_bytes,
                        shift, lane);
            cp_async_wait<0>();
            __syncwarp();
            const float pd = pair_distance<kFP32, kL2>(q, my_row, g.dim, row_bytes, half);
            __syncwarp();
            return lane < cnt ? pd : INFINITY;
        };
        // The links of `node` on `layer` into lbuf; returns how many were copied (cap).
        const auto load_links = [&](std::uint32_t node, std::uint32_t layer) {
            const std::uint32_t* src = block_of(a, node, layer);
            const std::uint32_t stride = layer == 0 ? g.stride0 : g.stride_up;
            for (std::uint32_t x = lane; x < stride; x += 32) {
                lbuf[x] = src[x];
            }
            __syncwarp();
            return layer == 0 ? g.cap0 : g.cap_up;
        };

        // The entry point and the greedy walk above the node's level.
        std::uint32_t cur = a.entry;
        if (lane == 0) {
            fresh[0] = cur;
        }
        __syncwarp();
        float curd = __shfl_sync(kFull, score(0, 1), 0);
        for (std::uint32_t layer = a.max_level; layer > top; --layer) {
            for (std::uint32_t hop = 0; hop <= g.n; ++hop) {
                const std::uint32_t cap = load_links(cur, layer);
                int f = 0;
                for (std::uint32_t c0 = 0; c0 < cap; c0 += 32) {
                    const std::uint32_t id = c0 + lane < cap ? lbuf[c0 + lane] : kNoId;
                    const bool valid = id != kNoId && id < g.n;
                    const std::uint32_t m = __ballot_sync(kFull, valid);
                    if (valid) {
                        fresh[f + __popc(m & ((1u << lane) - 1u))] = id;
                    }
                    f += __popc(m);
                }
                __syncwarp();
                float best_d = INFINITY;
                std::uint32_t best_i = 0xFFFFFFFFu;
                for (int s0 = 0; s0 < f; s0 += rounds_cap) {
                    const int cnt = min(rounds_cap, f - s0);
                    const float d = score(s0, cnt);
                    float bd;
                    std::uint32_t bi;
                    warp_argmin(d, lane < cnt ? static_cast<std::uint32_t>(s0 + lane) : 0xFFFFFFFFu, bd, bi);
                    if (bd < best_d) {
                        best_d = bd;
                        best_i = bi;
                    }
                }
                if (f > 0 && best_d < curd) {
                    cur = fresh[best_i];
                    curd = best_d;
                    __syncwarp();
                } else {
                    break;
                }
            }
        }

        // Candidate searches on the node's layers, top-down.
        for (int layer = static_cast<int>(top); layer >= 0; --layer) {
            for (std::uint32_t x = lane; x < a.hash_slots; x += 32) {
                table[x] = kNoId;
            }
            __syncwarp();
            if (lane == 0) {
                first_visit(table, hmask, cur);
                rd[0] = curd;
                rid[0] = cur;
            }
            __syncwarp();
            int r = 1;
            int scan = 0;
            const int ef = static_cast<int>(a.ef);
            for (std::uint32_t step = 0; step <= g.n; ++step) {
                const int p = first_unexpanded(rid, scan, r, lane);
                if (p >= r) {
                    break;
                }
                const std::uint32_t node = rid[p] & kIdMask;
                __syncwarp();
                if (lane == 0) {
                    rid[p] = node | kExpanded;
                }
                scan = p + 1;
                const std::uint32_t cap = load_links(node, static_cast<std::uint32_t>(layer));
                int f = 0;
                for (std::uint32_t c0 = 0; c0 < cap; c0 += 32) {
                    const std::uint32_t id = c0 + lane < cap ? lbuf[c0 + lane] : kNoId;
                    const bool present = id != kNoId && id < g.n;
                    const bool isnew = present && first_visit(table, hmask, id);
                    const std::uint32_t m = __ballot_sync(kFull, isnew);
                    if (isnew) {
                        fresh[f + __popc(m & ((1u << lane) - 1u))] = id;
                    }
                    f += __popc(m);
                }
                __syncwarp();
                for (int s0 = 0; s0 < f; s0 += rounds_cap) {
                    const int cnt = min(rounds_cap, f - s0);
                    const float d = score(s0, cnt);
                    const bool valid = lane < cnt;
                    const std::uint32_t id = valid ? fresh[s0 + lane] : kNoId;
                    __syncwarp();
                    unsigned long long unused = 0;
                    const int low = merge_round(rd, rid, r, ef, d, id, valid, ap, lane, unused);
                    scan = min(scan, low);
                }
            }
            const std::uint32_t slot = a.cand_at[i] + static_cast<std::uint32_t>(layer);
            for (int x = lane; x < r; x += 32) {
                a.cand_ids[static_cast<std::size_t>(slot) * a.efcap + x] = rid[x] & kIdMask;
                a.cand_d[static_cast<std::size_t>(slot) * a.efcap + x] = rd[x];
            }
            if (lane == 0) {
                a.cand_n[slot] = static_cast<std::uint32_t>(r);
            }
            cur = rid[0] & kIdMask;  // the next layer starts from the closest one found
            curd = rd[0];
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// 2. Neighbor selection, own lists, proposals. One warp per (node, layer) candidate list.

// Walking `cands` (sorted by closer) from the closest, keeps one when it is closer to the base
// than to every kept one, until `m` are kept; with m or fewer candidates all are kept
// (the heuristic of src/hnsw.cpp:395-421). kept_ids / kept_d in shared memory.
template <bool kL2>
__device__ int select_heuristic(const BuildArgs& a, const std::uint32_t* cand_ids,
                                const float* cand_d, int n_cand, int m, std::uint32_t* kept_ids,
                                float* kept_d, int lane) {
    if (n_cand <= m) {
        for (int x = lane; x < n_cand; x += 32) {
            kept_ids[x] = cand_ids[x];
            kept_d[x] = cand_d[x];
        }
        __syncwarp();
        return n_cand;
    }
    int kept = 0;
    for (int j = 0; j < n_cand && kept < m; ++j) {
        const std::uint32_t c = cand_ids[j];
        const float dc = cand_d[j];
        bool closer_to_kept = false;
        for (int s0 = 0; s0 < kept; s0 += 32) {
            const int s = s0 + lane;
            const bool hit = s < kept && vec_distance<kL2>(a, c, kept_ids[s]) < dc;
            closer_to_kept |= __any_sync(kFull, hit);
        }
        if (!closer_to_kept) {
            if (lane == 0) {
                kept_ids[kept] = c;
                kept_d[kept] = dc;
            }
            ++kept;
            __syncwarp();
        }
    }
    return kept;
}

template <bool kL2>
__global__ void __launch_bounds__(128) build_select_kernel(const BuildArgs a) {
    __shared__ std::uint32_t s_ids[4][64];
    __shared__ float s_d[4][64];
    const int lane = static_cast<int>(threadIdx.x & 31);
    const int warp = static_cast<int>(threadIdx.x >> 5);
    const std::uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (std::uint32_t i = blockIdx.x * (blockDim.x >> 5) + warp; i < a.count; i += warps) {
        const std::uint32_t v = a.first + i;
        const std::uint32_t level = a.levels[v];
        const std::uint32_t top = level < a.max_level ? level : a.max_level;
        for (std::uint32_t layer = 0; layer <= top; ++layer) {
            const std::uint32_t slot = a.cand_at[i] + layer;
            const int n_cand = static_cast<int>(a.cand_n[slot]);
            const int kept = select_heuristic<kL2>(a, a.cand_ids + static_cast<std::size_t>(slot) * a.efcap,
                                                   a.cand_d + static_cast<std::size_t>(slot) * a.efcap,
                                                   n_cand, static_cast<int>(a.M), s_ids[warp], s_d[warp],
                                                   lane);
            // The node's own list: the kept ones, closest first.
            std::uint32_t* own = block_of(a, v, layer);
            const std::uint32_t stride = layer == 0 ? a.g.stride0 : a.g.stride_up;
            for (std::uint32_t x = lane; x < stride; x += 32) {
                own[x] = static_cast<int>(x) < kept ? s_ids[warp][x] : kNoId;
            }
            // One proposal to each chosen neighbor.
            for (int x = lane; x < kept; x += 32) {
                const std::uint32_t list = list_of(a, s_ids[warp][x], layer);
                const std::uint32_t at = atomicAdd(a.prop_count + list, 1u);
                if (at == 0) {
                    a.touched[atomicAdd(a.touched_n, 1u)] = list;
                }
                if (at < kProposals) {
                    a.prop_ids[static_cast<std::size_t>(list) * kProposals + at] = v;
                    a.prop_d[static_cast<std::size_t>(list) * kProposals + at] = s_d[warp][x];
                }
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// 3. Links back. One warp per neighbor list that received proposals.

template <bool kL2>
__global__ void __launch_bounds__(128) build_link_kernel(const BuildArgs a) {
    constexpr int kMaxCand = 128 + kProposals;  // a full list (cap0 <= 128) plus the proposals
    __shared__ std::uint32_t s_ids[4][kMaxCand];
    __shared__ float s_d[4][kMaxCand];
    __shared__ std::uint32_t k_ids[4][128];
    __shared__ float k_d[4][128];
    const int lane = static_cast<int>(threadIdx.x & 31);
    const int warp = static_cast<int>(threadIdx.x >> 5);
    const std::uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const std::uint32_t touched = *a.touched_n;
    for (std::uint32_t t = blockIdx.x * (blockDim.x >> 5) + warp; t < touched; t += warps) {
        const std::uint32_t list = a.touched[t];
        const bool upper = list >= a.g.n;
        const std::uint32_t node = upper ? a.up_owner[list - a.g.n] : list;
        std::uint32_t* block = upper ? a.links_up + static_cast<std::size_t>(list - a.g.n) * a.g.stride_up
                                     : a.links0 + static_cast<std::size_t>(node) * a.g.stride0;
        const int cap = static_cast<int>(upper ? a.g.cap_up : a.g.cap0);
        const int props = static_cast<int>(min(a.prop_count[list], kProposals));
        int have = 0;  // existing links: a prefix of the block
        for (int c0 = 0; c0 < cap; c0 += 32) {
            const bool used = c0 + lane < cap && block[c0 + lane] != kNoId;
            have += __popc(__ballot_sync(kFull, used));
        }
        const std::uint32_t* pid = a.prop_ids + static_cast<std::size_t>(list) * kProposals;
        const float* pd = a.prop_d + static_cast<std::size_t>(list) * kProposals;
        if (have + props <= cap) {
            for (int x = lane; x < props; x += 32) {
                block[have + x] = pid[x];
            }
        } else {
            // Re-select from the old links (distances recomputed) plus the proposals, in closer
            // order: repeatedly take the closest remaining candidate.
            const int total = have + props;
            for (int x = lane; x < total; x += 32) {
                if (x < have) {
                    const std::uint32_t id = block[x];
                    s_ids[warp][x] = id;
                    s_d[warp][x] = vec_distance<kL2>(a, node, id);
                } else {
                    s_ids[warp][x] = pid[x - have];
                    s_d[warp][x] = pd[x - have];
                }
            }
            __syncwarp();
            int kept = 0;
            for (int step = 0; step < total && kept < cap; ++step) {
                float best_d = INFINITY;
                std::uint32_t best_id = kNoId;
                for (int x0 = 0; x0 < total; x0 += 32) {
                    const int x = x0 + lane;
                    const float d = x < total ? s_d[warp][x] : INFINITY;
                    const std::uint32_t id = x < total ? s_ids[warp][x] : kNoId;
                    float bd;
                    std::uint32_t bi;
                    warp_argmin(d, id, bd, bi);
                    if (closer(bd, bi, best_d, best_id)) {
                        best_d = bd;
                        best_id = bi;
                    }
                }
                if (best_id == kNoId) {
                    break;
                }
                // Remove it from the pool (every copy of that id; ids are unique per list).
                for (int x = lane; x < total; x += 32) {
                    if (s_ids[warp][x] == best_id) {
                        s_d[warp][x] = INFINITY;
                        s_ids[warp][x] = kNoId;
                    }
                }
                bool closer_to_kept = false;
                for (int s0 = 0; s0 < kept; s0 += 32) {
                    const int s = s0 + lane;
                    const bool hit = s < kept && vec_distance<kL2>(a, best_id, k_ids[warp][s]) < best_d;
                    closer_to_kept |= __any_sync(kFull, hit);
                }
                if (!closer_to_kept) {
                    if (lane == 0) {
                        k_ids[warp][kept] = best_id;
                        k_d[warp][kept] = best_d;
                    }
                    ++kept;
                }
                __syncwarp();
            }
            for (int x = lane; x < cap; x += 32) {
                block[x] = x < kept ? k_ids[warp][x] : kNoId;
            }
        }
        __syncwarp();
        if (lane == 0) {
            a.prop_count[list] = 0;
        }
    }
}

std::uint32_t round_up32(std::uint32_t x, std::uint32_t m) { return (x + m - 1) / m * m; }

}  // namespace
}  // namespace vdx::dev

namespace vdx {

void HnswIndex::add_gpu(MatrixView<float> vectors, int device) {
    detail::check_new_vectors("HnswIndex::add", {metric_, dim(), size()}, vectors.dim(), vectors.data());
    if (params_.M > 64) {
        throw std::invalid_argument("HnswIndex::add_gpu: the GPU build supports M up to 64");
    }
    invalidate_device();
    const std::size_t first = size();
    const std::size_t total = first + vectors.rows();
    if (total >= (std::size_t{1} << 31)) {
        throw std::length_error("HnswIndex::add_gpu: at most 2^31 - 1 nodes");
    }
    vectors_.reserve_rows(total);
    levels_.reserve(total);
    layer0_.reserve(total * (1 + max_links(0)));
    upper_.reserve(total);
    // Every vector stored (levels drawn in the serial order) before anything is linked.
    for (std::size_t r = 0; r < vectors.rows(); ++r) {
        append_node(vectors.row(r));
    }
    // The first nodes one by one on the host, exactly as the serial build.
    std::size_t next = first;
    const std::size_t seed_end = std::min(total, std::max<std::size_t>(first, dev::kSeedNodes));
    for (; next < seed_end; ++next) {
        link_serial(static_cast<Id>(next));
    }
    if (next == total) {
        return;
    }

    // The device mirror of everything stored (unlinked nodes have empty lists), grown in place.
    const DeviceGraph& dgc = device_graph(device, Precision::FP32);
    auto& dg = const_cast<DeviceGraph&>(dgc);
    gpu::use_device(device);
    gpu::Workspace& ws = gpu::workspace(device);
    cudaStream_t stream = ws.stream;
    const std::uint32_t n = dg.view.n;
    const std::uint32_t n_up = static_cast<std::uint32_t>(
        std::accumulate(levels_.begin(), levels_.end(), std::size_t{0}));

    // Per-run device buffers.
    struct Buf {
        void* p = nullptr;
        ~Buf() {
            if (p != nullptr) {
                cudaFree(p);
            }
        }
    };
    const auto alloc = [](Buf& b, std::size_t bytes, const char* what) {
        b.p = gpu::device_alloc(std::max<std::size_t>(bytes, 4), what);
    };
    Buf d_levels, d_owner, d_prop_count, d_prop_ids, d_prop_d, d_touched, d_small, d_cand_at, d_cand_ids,
        d_cand_d, d_cand_n;
    alloc(d_levels, n, "levels");
    gpu::check(cudaMemcpyAsync(d_levels.p, levels_.data(), n, cudaMemcpyHostToDevice, stream), "levels");
    {
        std::vector<std::uint32_t> owner(n_up);
        std::size_t at = 0;
        for (std::uint32_t i = 0; i < n; ++i) {
            for (std::uint32_t l = 0; l < levels_[i]; ++l) {
                owner[at++] = i;
            }
        }
        alloc(d_owner, n_up * 4ull, "upper owners");
        gpu::check(cudaMemcpy(d_owner.p, owner.data(), n_up * 4ull, cudaMemcpyHostToDevice), "owners");
    }
    const std::size_t lists = static_cast<std::size_t>(n) + n_up;
    alloc(d_prop_count, lists * 4, "proposal counts");
    alloc(d_prop_ids, lists * dev::kProposals * 4, "proposals");
    alloc(d_prop_d, lists * dev::kProposals * 4, "proposal distances");
    alloc(d_touched, lists * 4, "touched lists");
    alloc(d_small, 256, "build counters");
    gpu::check(cudaMemsetAsync(d_prop_count.p, 0, lists * 4, stream), "proposal counts");

    dev::BuildArgs a{};
    a.g = dg.view;
    a.links0 = static_cast<std::uint32_t*>(dg.links0_alloc);
    a.links_up = static_cast<std::uint32_t*>(dg.links_up_alloc);
    a.levels = static_cast<const std::uint8_t*>(d_levels.p);
    a.up_owner = static_cast<const std::uint32_t*>(d_owner.p);
    a.n_up = n_up;
    a.M = static_cast<std::uint32_t>(params_.M);
    a.ef = static_cast<std::uint32_t>(std::max(params_.ef_construction, params_.M));
    a.efcap = 32;
    while (a.efcap < a.ef) {
        a.efcap <<= 1;
    }
    a.hash_slots = 2048;
    while (a.hash_slots < 16 * a.efcap && a.hash_slots < 16384) {
        a.hash_slots <<= 1;
    }
    a.rows_cap = std::min<std::uint32_t>(16, std::max<std::uint32_t>(1, dg.view.cap0));
    a.prop_count = static_cast<std::uint32_t*>(d_prop_count.p);
    a.prop_ids = static_cast<std::uint32_t*>(d_prop_ids.p);
    a.prop_d = static_cast<float*>(d_prop_d.p);
    a.touched = static_cast<std::uint32_t*>(d_touched.p);
    a.touched_n = static_cast<std::uint32_t*>(d_small.p);
    a.claim = static_cast<std::uint32_t*>(d_small.p) + 1;
    // Per-warp shared memory of the search kernel.
    {
        std::uint32_t off = dev::round_up32(dg.view.row32 * 4, 16);
        a.off_r = off;
        off += dev::round_up32(a.efcap * 8, 16);
        a.off_hash = off;
        off += a.hash_slots * 4;
        a.off_links = off;
        off += dev::round_up32(std::max(dg.view.stride0, dg.view.stride_up) * 4, 16);
        a.off_rows = off;
        off += dev::round_up32(a.rows_cap * dev::padded_row_stride(dg.view.row32 * 4), 16);
        a.off_fresh = off;
        off += dev::round_up32(std::max<std::uint32_t>(dg.view.cap0, 32) * 4, 16);
        a.off_ap = off;
        off += 32 * 4;
        a.warp_bytes = dev::round_up32(off, 16);
    }
    const std::size_t smem = static_cast<std::size_t>(a.warp_bytes) * dev::kBuildWarps;
    const bool l2 = metric_ == Metric::L2;
    auto* search = l2 ? &dev::build_search_kernel<true> : &dev::build_search_kernel<false>;
    auto* select = l2 ? &dev::build_select_kernel<true> : &dev::build_select_kernel<false>;
    auto* link = l2 ? &dev::build_link_kernel<true> : &dev::build_link_kernel<false>;
    gpu::check(cudaFuncSetAttribute(search, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)), "build smem");
    int sms = 0, per_sm = 0;
    gpu::check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sms");
    gpu::check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, search, dev::kBuildWarps * 32, smem),
               "occupancy");
    const int search_blocks = sms * std::max(per_sm, 1);

    std::vector<std::uint32_t> cand_at;
    std::size_t cand_cap = 0;
    Id entry = entry_point_;
    std::size_t max_level = max_level_;
    while (next < total) {
        // The batch: a 32nd of the graph (at least 32, at most 8192); a node that raises the top
        // layer closes its batch.
        std::size_t end = std::min(total, next + std::clamp<std::size_t>(next / 32, 32, dev::kMaxBatch));
        for (std::size_t v = next; v < end; ++v) {
            if (levels_[v] > max_level) {
                end = v + 1;
                break;
            }
        }
        const std::uint32_t count = static_cast<std::uint32_t>(end - next);
        cand_at.resize(count);
        std::uint32_t slots = 0;
        for (std::uint32_t i = 0; i < count; ++i) {
            cand_at[i] = slots;
            slots += 1 + std::min<std::uint32_t>(levels_[next + i], static_cast<std::uint32_t>(max_level));
        }
        if (slots > cand_cap || d_cand_at.p == nullptr) {
            cand_cap = std::max<std::size_t>(slots, 2 * cand_cap);
            for (Buf* b : {&d_cand_ids, &d_cand_d, &d_cand_n, &d_cand_at}) {
                if (b->p != nullptr) {
                    gpu::check(cudaStreamSynchronize(stream), "build buffers");
                    cudaFree(b->p);
                    b->p = nullptr;
                }
            }
            alloc(d_cand_ids, cand_cap * a.efcap * 4, "candidates");
            alloc(d_cand_d, cand_cap * a.efcap * 4, "candidate distances");
            alloc(d_cand_n, cand_cap * 4, "candidate counts");
            alloc(d_cand_at, std::max<std::size_t>(cand_cap, dev::kMaxBatch) * 4, "candidate slots");
        }
        gpu::check(cudaMemcpyAsync(d_cand_at.p, cand_at.data(), count * 4ull, cudaMemcpyHostToDevice, stream),
                   "candidate slots");
        gpu::check(cudaStreamSynchronize(stream), "candidate slots");  // cand_at is reused next batch
        a.first = static_cast<std::uint32_t>(next);
        a.count = count;
        a.entry = entry;
        a.max_level = static_cast<std::uint32_t>(max_level);
        a.cand_at = static_cast<const std::uint32_t*>(d_cand_at.p);
        a.cand_ids = static_cast<std::uint32_t*>(d_cand_ids.p);
        a.cand_d = static_cast<float*>(d_cand_d.p);
        a.cand_n = static_cast<std::uint32_t*>(d_cand_n.p);
        gpu::check(cudaMemsetAsync(d_small.p, 0, 8, stream), "build counters");
        search<<<std::min<int>(search_blocks, static_cast<int>((count + dev::kBuildWarps - 1) / dev::kBuildWarps)),
                 dev::kBuildWarps * 32, smem, stream>>>(a);
        gpu::check(cudaGetLastError(), "build search");
        const int sel_blocks = std::min<int>(sms * 8, static_cast<int>((count + 3) / 4));
        select<<<sel_blocks, 128, 0, stream>>>(a);
        gpu::check(cudaGetLastError(), "build select");
        link<<<sms * 8, 128, 0, stream>>>(a);
        gpu::check(cudaGetLastError(), "build link");
        if (levels_[end - 1] > max_level) {
            max_level = levels_[end - 1];
            entry = static_cast<Id>(end - 1);
        }
        next = end;
    }
    gpu::check(cudaStreamSynchronize(stream), "build");

    // The graph back into the host layout: [count, ids...] blocks.
    {
        const std::size_t cap0 = max_links(0);
        std::vector<std::uint32_t> dev0(static_cast<std::size_t>(n) * dg.view.stride0);
        gpu::check(cudaMemcpy(dev0.data(), dg.links0_alloc, dev0.size() * 4, cudaMemcpyDeviceToHost),
                   "download links");
        for (std::size_t v = first; v < total; ++v) {
            Id* block = this->block(static_cast<Id>(v), 0).data();
            std::uint32_t c = 0;
            for (; c < cap0 && dev0[v * dg.view.stride0 + c] != dev::kNoId; ++c) {
                block[1 + c] = dev0[v * dg.view.stride0 + c];
            }
            block[0] = c;
        }
        // Old nodes' lists changed too (links back): copy every layer-0 list.
        for (std::size_t v = 0; v < first; ++v) {
            Id* block = this->block(static_cast<Id>(v), 0).data();
            std::uint32_t c = 0;
            for (; c < cap0 && dev0[v * dg.view.stride0 + c] != dev::kNoId; ++c) {
                block[1 + c] = dev0[v * dg.view.stride0 + c];
            }
            block[0] = c;
        }
        if (n_up > 0) {
            std::vector<std::uint32_t> devu(static_cast<std::size_t>(n_up) * dg.view.stride_up);
            gpu::check(cudaMemcpy(devu.data(), dg.links_up_alloc, devu.size() * 4, cudaMemcpyDeviceToHost),
                       "download upper links");
            std::size_t b = 0;
            for (std::size_t v = 0; v < n; ++v) {
                for (std::size_t l = 1; l <= levels_[v]; ++l, ++b) {
                    Id* block = this->block(static_cast<Id>(v), l).data();
                    std::uint32_t c = 0;
                    for (; c < params_.M && devu[b * dg.view.stride_up + c] != dev::kNoId; ++c) {
                        block[1 + c] = devu[b * dg.view.stride_up + c];
                    }
                    block[0] = c;
                }
            }
        }
    }
    entry_point_ = entry;
    max_level_ = max_level;
    // The FP32 device mirror was built in place; its entry and top layer are now the host's,
    // and its upper copy is made from the finished upper layers.
    dg.view.entry = entry_point_;
    dg.view.max_level = static_cast<std::uint32_t>(max_level_);
    gpu::attach_upper_copy(*this, dg, stream);
}

}  // namespace vdx
