#pragma once

// Launch interface of the HNSW search kernels (search.cu).

#include <cuda_runtime.h>

#include <cstdint>

#include "vdx/device.hpp"

namespace vdx::dev {

// Per-launch device counters (stats[i], atomically accumulated over the launch).
enum Stat : int {
    kStatQueries = 0,     // queries searched
    kStatExpansions,      // layer-0 nodes expanded
    kStatDist0,           // layer-0 distance evaluations (traversal precision)
    kStatDistUpper,       // upper-layer distance evaluations, entry point included
    kStatLinkBytes,       // link-block bytes read: 4 * (1 + count) per block (algorithmic)
    kStatRowBytes,        // vector bytes gathered for distances (traversal rows, algorithmic)
    kStatRerankBytes,     // FP32 row bytes read by the re-rank
    kStatDuplicates,      // rediscovered nodes dropped by the merge (visited-filter misses)
    kStatPrefetchHits,    // expansions whose link block was already prefetched
    kStatLearnedStops,    // queries stopped by the learned criterion
    kStatCount
};

// Error codes written to status[0]; status[1] receives the lowest failing query row.
enum SearchError : std::uint32_t {
    kErrNone = 0,
    kErrNonFinite = 1,     // a query component is NaN or infinite
    kErrZeroCosine = 2,    // a cosine query cannot be normalized
    kErrBounds = 3,        // a link id out of range (a corrupted device graph)
    kErrCapacity = 4,      // ef exceeds the launch's result-list capacity
    kErrTimeout = 5,       // a bounded device wait gave up (tensor-core brute force)
};

// The learned early-termination network (12 -> 64 -> 64 -> 1, ReLU, sigmoid), as the search
// kernel reads it: BF16 weights, FP32 feature standardization and random projections.
struct StopNetView {
    const std::uint16_t* w1;   // [64][12] bf16 bits
    const std::uint16_t* w2;   // [64][64]
    const std::uint16_t* w3;   // [64]
    const float* b1;           // [64]
    const float* b2;           // [64]
    const float* b3;           // [1]
    const float* mean;         // [12] feature standardization
    const float* inv_std;      // [12]
    const float* proj;         // [4][dim] random projection rows
};

// Training-trace output: every 8 expansions a query's 12 features and its current top-k hits
// against `truth` are recorded (trace mode only).
struct TraceArgs {
    const std::uint32_t* truth;     // [nq][truth_k] ground-truth ids, or null (no tracing)
    std::uint32_t truth_k;
    std::uint32_t max_points;       // trace points per query
    float* features;                // [nq][max_points][12]
    std::uint8_t* hits;             // [nq][max_points] |current top-k ∩ truth|
    std::uint32_t* points;          // [nq] trace points written
    std::uint8_t* final_hits;       // [nq]
};

struct SearchArgs {
    DeviceGraphView g{};
    const float* queries = nullptr;       // nq rows of qstride floats
    std::uint32_t nq = 0;
    std::uint32_t qstride = 0;
    const std::uint32_t* nq_device = nullptr;   // batch size read on the device (<= nq) when non-null
    const std::uint32_t* k_per_q = nullptr;
    const std::uint32_t* ef_per_q = nullptr;
    std::uint32_t k = 10;
    std::uint32_t ef = 64;
    std::uint32_t out_stride = 10;         // entries per result row (>= every k)
    std::uint32_t* out_ids = nullptr;
    float* out_dists = nullptr;
    std::uint32_t* out_counts = nullptr;
    std::uint32_t* status = nullptr;       // 2 words, zeroed before launch
    unsigned long long* stats = nullptr;   // kStatCount words or null
    std::uint32_t* claim = nullptr;        // work counter, zeroed before launch
    std::uint32_t rerank = 0;              // re-score this many best in FP32 (0: none)
    std::uint32_t rerank_per_k = 0;        // non-zero: re-score rerank_per_k * k (rerank >= the
                                           // largest such width, for the scratch sizing)
    StopNetView stop{};
    const void* stop_enabled = nullptr;    // non-null: learned early termination is on
    unsigned long long* gvisited = nullptr; // global visited tables, one per warp (or null)
    std::uint32_t* gepoch = nullptr;        // per-warp query epoch counters
    std::uint32_t gslots = 0;               // slots a query uses (power of two, <= gstride)
    std::uint32_t gstride = 0;              // slots between two warps' tables
    std::uint32_t gwarps = 0;               // warps the tables were sized for
    float stop_threshold = 0.5F;
    std::uint32_t stop_min_hops = 16;
    // The network is consulted at a checkpoint only when the k-th distance has been unchanged
    // for this many expansions in a row (0 to 3; 0 consults it at every checkpoint).
    std::uint32_t stop_gate = 0;
    TraceArgs trace{};
    // Ordered launch (all three non-null, nq words each): a descent pass writes each query's
    // layer-0 entry (id, distance; id 0xFFFFFFFF for a query that failed its checks), the queries
    // are ordered by that distance, farthest first, and the layer-0 pass claims them in that
    // order, so the queries that will take longest start first and the grid's tail is short.
    std::uint32_t* entry_ids = nullptr;
    float* entry_d = nullptr;
    std::uint32_t* order = nullptr;
    std::uint32_t pass = 0;                // set by launch_search: 0 whole search, 1 descent,
                                           // 2 layer 0 from the entries, in `order`
    // Per-warp shared-memory layout (bytes), filled by plan_search().
    std::uint32_t efcap = 0, hash_slots = 0, rows_cap = 0, warp_bytes = 0;
    std::uint32_t off_r = 0, off_hash = 0, off_links = 0, off_rows = 0, off_fresh = 0, off_ap = 0;
    std::uint32_t off_hist = 0;
};

// Shape of one launch: warps per block and the per-warp buffers.
struct SearchPlan {
    int warps_per_block = 4;
    std::uint32_t efcap = 64;        // result-list capacity (>= every effective ef)
    std::uint32_t hash_slots = 2048; // visited-filter slots in shared memory (power of two)
    std::uint32_t global_slots = 0;  // > 0: the visited filter is a per-warp global table of
                                     // this many 8-byte slots (power of two) instead
    std::uint32_t rows_cap = 32;     // rows gathered per round
    int blocks = 0;                  // 0: as many as fit on the device
};

// Fills the layout fields of `args` for `plan`; returns the dynamic shared memory per block.
std::size_t plan_search(SearchArgs& args, const SearchPlan& plan);

// The default plan for a graph and the largest effective ef of a batch. allow_global: the caller
// can provide global visited tables (global_visited_bytes), used from ef capacity 512 up.
SearchPlan default_plan(const DeviceGraphView& g, std::uint32_t max_ef, bool allow_global = false);

// The most warps per block a plan of result capacity `efcap` may use on graph `g` (4 for the
// register-limited BF16 / FP8 kernels of capacity <= 64, else 8); launch_search rejects more.
int max_warps_per_block(const DeviceGraphView& g, std::uint32_t efcap);

// Warps the launch of `plan` runs (the grid the launcher picks before trimming it to a short
// batch), and the bytes of global visited tables and epoch counters for `warps` warps of
// `stride` slots each. A buffer is zeroed once when laid out; it stays valid for every later
// launch on one stream whose plan needs at most `stride` slots and `warps` warps (each warp's
// table and epoch counter keep their place, and epochs only grow).
std::uint32_t search_warps(SearchArgs& args, const SearchPlan& plan);
std::size_t global_visited_bytes(std::uint32_t stride, std::uint32_t warps);
// Points args at a global visited buffer laid out for `warps` warps of `stride` slots.
void bind_global_visited(SearchArgs& args, const SearchPlan& plan, void* buffer,
                         std::uint32_t stride, std::uint32_t warps);

// Launches the search for args.nq queries on `stream` (status, claim, claim + 1 and stats must
// be zeroed on that stream first): one kernel, or with entry_ids / entry_d / order set the
// ordered three (descent pass, order_kernel, layer-0 pass). Returns the CUDA error of the
// launches.
cudaError_t launch_search(SearchArgs& args, const SearchPlan& plan, cudaStream_t stream);

// Kernels launched by this thread's last launch_search (for launch accounting).
int search_kernels_per_launch();

}  // namespace vdx::dev
