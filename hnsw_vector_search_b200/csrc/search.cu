// HNSW search on the GPU: one warp per query, persistent blocks claiming queries from a counter.
//
// Per query (the reference's search_unchecked, src/hnsw.cpp:504-522):
//   1. load the query into shared memory, reject NaN/inf, normalize under cosine
//      (sqrt of the kernel-order <q, q>, IEEE division; src/vector_ops.cpp:14-34);
//   2. greedy descent over layers max_level..1 (src/hnsw.cpp:416-431): all links of the current
//      node are scored at once and the walk moves to the first strict minimum in link order,
//      which is exactly where the reference's sequential running-minimum scan ends;
//   3. the layer-0 beam (src/hnsw.cpp:438-482) over a sorted result list R of at most ef entries,
//      each with an "expanded" bit: repeatedly expand the closest unexpanded entry, score its
//      unvisited neighbors, and set R = top-ef(R + scored). This returns exactly the reference's
//      result: admitting a batch is the same as admitting one at a time (both keep the top ef of
//      everything scored), and the reference's candidate heap only ever matters through entries
//      still in R (a popped candidate evicted from R ends the search at the same point where R
//      has no unexpanded entry left).
//   4. write the first min(k, |R|) entries, closest first (ties by smaller id).
//
// Memory traffic: each expansion reads one link block (one 128-byte line at M = 16) and gathers
// the unvisited neighbors' rows with 16-byte cp.async copies into shared memory, all rows of a
// round in flight together; the link block of the next expansion, predicted exactly before the
// merge (the closer of R's first unexpanded entry and the round's best admissible candidate), is
// prefetched while the merge runs. The kernel is bound by the latency of that dependent chain
// per expansion and by instruction issue, not by DRAM bandwidth; the rest of this file keeps the
// chain short (register result list, bucketed filter, ballot merge, unrolled d = 128 distances)
// and the registers few (one kernel per pass and per learned-stop use).
//
// The visited set is a per-warp shared-memory open-addressing hash of 4-slot buckets (one 16-byte
// load per bucket, first_visit_bucket). It never reports an unvisited node as visited. If its
// probe limit is reached it reports "unvisited" and the node is scored again; the merge then drops
// the copy already in R (equal distance and id), so results stay exact and the only cost is the
// extra row read (counted in kStatDuplicates).
//
// Every loop is bounded (the walk cannot run longer than the node count), and no kernel waits on
// another thread or block: cp.async completion is a hardware wait.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <type_traits>
#include <vector>

#include "beam.cuh"
#include "common.cuh"
#include "search.cuh"

namespace vdx::dev {
namespace {

struct Counters {
    unsigned long long v[kStatCount];
};

__device__ __forceinline__ void report(std::uint32_t* status, std::uint32_t code,
                                       std::uint32_t row) {
    atomicCAS(status, 0u, code);
    atomicMin(status + 1, row);
}

// The same filter in global memory, for large ef (a per-warp table too big for shared memory):
// 64-bit slots hold (query epoch << 32 | id); a slot whose epoch is not the current query's is
// empty, so the table never needs clearing between queries. Like first_visit_bucket the table
// is read as 4-slot buckets (32 bytes, two 16-byte L2 loads): an id lives in the first bucket of
// its sequence that had an empty slot when it was inserted, and within a query slots only fill.
// Only this warp's lanes write its table, so a claimed slot is lost only to a lane of the same
// warp (then the bucket is read again); a lane that meets kProbes / 4 full buckets reports
// "unvisited". Every loop is bounded.
__device__ __forceinline__ bool first_visit_global(unsigned long long* table, std::uint32_t mask,
                                                   std::uint32_t id, std::uint32_t epoch) {
    const unsigned long long key = (static_cast<unsigned long long>(epoch) << 32) | id;
    std::uint32_t b = (id * 2654435761u) & mask & ~3u;
    int full = 0;
#pragma unroll 1
    for (int step = 0; step < 2 * kProbes; ++step) {
        const ulonglong2 lo = __ldcg(reinterpret_cast<const ulonglong2*>(table + b));
        const ulonglong2 hi = __ldcg(reinterpret_cast<const ulonglong2*>(table + b + 2));
        const unsigned long long v[4] = {lo.x, lo.y, hi.x, hi.y};
        if (v[0] == key || v[1] == key || v[2] == key || v[3] == key) {
            return false;
        }
        int e = 4;
#pragma unroll
        for (int i = 3; i >= 0; --i) {
            e = static_cast<std::uint32_t>(v[i] >> 32) != epoch ? i : e;
        }
        if (e < 4) {
            const unsigned long long old = e == 0 ? v[0] : e == 1 ? v[1] : e == 2 ? v[2] : v[3];
            const unsigned long long prev = atomicCAS(table + b + e, old, key);
            if (prev == old) {
                return true;
            }
            if (prev == key) {
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


// ---------------------------------------------------------------------------------------------
// Learned early termination: features and the network, evaluated by a whole warp (every lane
// computes the same features from shared memory; the two hidden layers spread over the lanes).

constexpr int kFeatures = 12;
constexpr int kHidden = 64;
constexpr int kHist = 8;   // ring of the k-th distance after every 4th expansion

__device__ __forceinline__ float sgnlog(float x) { return copysignf(log1pf(fabsf(x)), x); }

// The 12 features of a query's search state after `hops` expansions (the model's inputs):
//   0 log(1 + |q|)                      1 signed log of the layer-0 entry distance
//   2 log(1 + (d_k - d_1) / |d_1|)      3..5 relative drop of d_k over the last 4 / 8 / 16
//   6 log(1 + hops)                     7 log(1 + expansions since d_k last changed, <= 31)
//   8..11 query projections
// None depends on ef, so a model trained on traces at one ef cap reads the same features at
// another. Called by every lane (the ballot of feature 7 needs the whole warp).
// `fc` holds the query's constant features: [0] |q|, [1] layer-0 entry distance, [2..5] the
// projections.
// `ring` holds d_k after every 4th expansion (ring[(h / 4) % 8] after expansion h, h > 0), and
// `unchanged` counts the expansions since d_k last changed (a candidate kept at a position below
// k), so the walk writes shared memory only every 4th expansion.
__device__ __forceinline__ void stop_features(float* f, const float* fc, const float* rd, int r,
                                              int k, const float* ring, int hops, int unchanged) {
    const float qlen = fc[0];
    const float d_entry = fc[1];
    const int kk = r < k ? r : k;
    const float d1 = rd[0];
    const float dk = rd[kk - 1];
    f[0] = log1pf(qlen);
    f[1] = sgnlog(d_entry);
    f[2] = log1pf(fmaxf(dk - d1, 0.0F) / (fabsf(d1) + 1e-3F * (1.0F + fabsf(dk))));
    const int ws[3] = {4, 8, 16};
#pragma unroll
    for (int w = 0; w < 3; ++w) {
        const int back = hops - ws[w] > 4 ? hops - ws[w] : 4;  // the earliest sample is after 4
        const float prev = ring[(back >> 2) & 7];
        const float drop = (prev - dk) / (fabsf(dk) + 1e-6F * (1.0F + fabsf(dk)));
        f[3 + w] = fminf(fmaxf(drop, -10.0F), 10.0F);
    }
    f[6] = log1pf(static_cast<float>(hops));
    f[7] = log1pf(static_cast<float>(unchanged < 31 ? unchanged : 31));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        f[8 + i] = fc[2 + i];
    }
}


// P(converged) of the network for features f (identical in every lane); h1 is 64 floats of
// per-warp shared scratch. Lane L computes hidden units L and L + 32 of both layers from the
// packed bf16 pairs (see upload_stop_net), the two chains side by side in the same order as a
// unit-by-unit evaluation.
__device__ __forceinline__ float stop_probability(const StopNetView& net, const float* f, float* h1,
                                                  int lane) {
    float x[kFeatures];
#pragma unroll
    for (int c = 0; c < kFeatures; ++c) {
        x[c] = (f[c] - net.mean[c]) * net.inv_std[c];
    }
    const uint4* w1 = reinterpret_cast<const uint4*>(net.w1) + lane * (kFeatures / 4);
    float a0 = net.b1[lane];
    float a1 = net.b1[lane + 32];
#pragma unroll
    for (int c4 = 0; c4 < kFeatures / 4; ++c4) {
        const uint4 w = __ldg(w1 + c4);
        const std::uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a0 = fmaf(__uint_as_float(ws[u] << 16), x[4 * c4 + u], a0);
            a1 = fmaf(__uint_as_float(ws[u] & 0xFFFF0000u), x[4 * c4 + u], a1);
        }
    }
    __syncwarp();
    h1[lane] = fmaxf(a0, 0.0F);
    h1[lane + 32] = fmaxf(a1, 0.0F);
    __syncwarp();
    float z0 = net.b2[lane];
    float z1 = net.b2[lane + 32];
    const uint4* w2 = reinterpret_cast<const uint4*>(net.w2) + lane;
#pragma unroll 4
    for (int g4 = 0; g4 < kHidden / 4; ++g4) {
        const uint4 w = __ldg(w2 + g4 * 32);
        const float4 h = *reinterpret_cast<const float4*>(h1 + 4 * g4);
        const std::uint32_t ws[4] = {w.x, w.y, w.z, w.w};
        const float hs[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            z0 = fmaf(__uint_as_float(ws[u] << 16), hs[u], z0);
            z1 = fmaf(__uint_as_float(ws[u] & 0xFFFF0000u), hs[u], z1);
        }
    }
    const std::uint32_t w3 = reinterpret_cast<const std::uint32_t*>(net.w3)[lane];
    float part = __uint_as_float(w3 << 16) * fmaxf(z0, 0.0F) +
                 __uint_as_float(w3 & 0xFFFF0000u) * fmaxf(z1, 0.0F);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        part += __shfl_xor_sync(kFull, part, o);
    }
    const float logit = part + net.b3[0];
    return 1.0F / (1.0F + __expf(-logit));
}

// The learned stop's decision at a checkpoint of a stop-only kernel: the features and the
// network, called out of line so that the walk around it keeps the register allocation of the
// plain kernels (the network's accumulators and weight loads would otherwise compete with the
// walk's registers in every expansion). Every lane returns the same answer.
__device__ __noinline__ bool stop_decision(const StopNetView net, const float* fc, const float* rd,
                                           int r, int k, const float* ring, int hops, int unchanged,
                                           float* h1, float threshold, int lane) {
    float f[kFeatures];
    stop_features(f, fc, rd, r, k, ring, hops, unchanged);
    return stop_probability(net, f, h1, lane) >= threshold;
}

// Launch bounds. The register-beam kernels over BF16 / FP8 rows need ~10 KB of shared memory
// per warp, room for 20 resident warps per SM, but at the 128 registers the compiler picks under
// 256 threads only 16 fit: they are held to 96 registers (blocks of at most 4 warps, 5 per SM;
// 5-6 % faster at ef 36-64 on the 1M x 128 workload, results identical). The others are bound
// by shared memory before registers and keep the compiler's choice (minimum blocks 0: none).
template <int P, bool kRegR>
constexpr bool kLowRegs = kRegR && P != kFP32;
template <int P, bool kRegR>
constexpr int kMaxThreads = kLowRegs<P, kRegR> ? 128 : 256;

// pair_distance with the loops of the most common dimension (128, SIFT-like data) unrolled at
// compile time; any other dimension takes the general loop. Same bits either way.
template <int P, bool kL2>
__device__ __forceinline__ float row_distance(const float* q, const unsigned char* row,
                                              std::uint32_t dim, std::uint32_t row_bytes, int half) {
    return dim == 128 ? pair_distance<P, kL2, 128>(q, row, dim, row_bytes, half)
                      : pair_distance<P, kL2>(q, row, dim, row_bytes, half);
}

// The distances of a round of `cnt` staged rows (warp-uniform), valid in lane r for row r: at
// dimension 128 a round of at most 8 FP32 / BF16 rows is scored by four lanes a row
// (quad_distance, row lane & 7), every other round by two (row_distance, row lane & 15). Same
// bits either way. Rows past the round re-read the buffer's last row (results masked).
template <int P, bool kL2>
__device__ __forceinline__ float round_distance(const float* q, const unsigned char* rows,
                                                std::uint32_t stride, const unsigned char* my_row,
                                                std::uint32_t dim, std::uint32_t row_bytes, int half,
                                                int lane, int cnt, int rows_cap) {
    if constexpr (P != kFP8) {
        if (dim == 128 && cnt <= 8) {
            const int row = min(lane & 7, rows_cap - 1);
            return quad_distance<P, kL2, 128>(q, rows + static_cast<std::uint32_t>(row) * stride,
                                              lane >> 3);
        }
    }
    return row_distance<P, kL2>(q, my_row, dim, row_bytes, half);
}

// Which learned-termination code a search kernel carries: none (plain searches), the stop only,
// or the stop and the training traces.
enum LearnMode : int { kLearnNone = 0, kLearnStop = 1, kLearnTrace = 2 };

// kRegR: R in registers (RegBeam, result capacity up to 64) instead of shared memory.
// kLearn: the learned-termination code compiled in (LearnMode; the variants launch only when the
// stop or tracing is on, so plain searches carry neither the code nor its registers, BF16 ef 36
// 7 % faster, and a stopping search does not carry the trace writer). Without that code the
// compiler's own register target for the shared-memory-beam kernels fell to 80 with spills, so
// those are bounded like the rest at 128 (2 blocks of 256).
// kPass: the pass compiled (0 the whole search, 1 the descent of an ordered launch, 2 its layer-0
// pass), so each kernel carries only the code its pass runs.
template <int P, bool kL2, bool kRegR, int kLearn, int kPass>
__global__ void __launch_bounds__(kMaxThreads<P, kRegR>,
                                  kLowRegs<P, kRegR> ? 5 : (kLearn != kLearnNone ? 0 : 2))
    search_kernel(const SearchArgs a) {
    constexpr std::uint32_t pass = kPass;
    // Ordered launch: order_kernel and the layer-0 pass are launched as programmatic dependents
    // (they may start while the kernel before them finishes); the descent lets its dependent
    // launch at once, and the layer-0 pass waits in hardware until order_kernel has completed
    // and its writes are visible. Without that launch attribute the wait returns at once.
    if constexpr (kPass == 1) {
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    }
    if constexpr (kPass == 2) {
        asm volatile("griddepcontrol.wait;" ::: "memory");
    }
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
    float* hist = reinterpret_cast<float*>(ws + a.off_hist);  // kHist sampled k-th distances
    float* h1 = hist + kHist;                                 // kHidden network scratch
    float* fc = h1 + kHidden;                                 // the query's constant features

    const DeviceGraphView& g = a.g;
    const bool learned = kLearn != kLearnNone && a.stop_enabled != nullptr;
    const bool tracing = kLearn == kLearnTrace && a.trace.truth != nullptr;
    const auto* vecs = static_cast<const unsigned char*>(g.vectors);
    // A device-side batch size never exceeds the buffers' capacity (a.nq).
    const std::uint32_t nq = a.nq_device != nullptr ? min(*a.nq_device, a.nq) : a.nq;
    const std::uint32_t hmask = a.hash_slots - 1;
    // With a global visited filter each warp of the grid owns one table and one epoch counter.
    const std::uint32_t gwarp = blockIdx.x * (blockDim.x >> 5) + static_cast<std::uint32_t>(warp);
    unsigned long long* const gtable =
        a.gvisited != nullptr ? a.gvisited + static_cast<std::size_t>(gwarp) * a.gstride : nullptr;
    const std::uint32_t gmask = a.gslots - 1;
    const auto visit = [&](std::uint32_t id, std::uint32_t epoch) {
        return gtable != nullptr ? first_visit_global(gtable, gmask, id, epoch)
                                 : first_visit_bucket(table, hmask, id);
    };
    // Two lanes score each row (pair_distance), so a round stages at most 16 rows.
    const int rounds_cap = static_cast<int>(a.rows_cap < 16 ? a.rows_cap : 16);
    const std::uint32_t stride_s = padded_row_stride(g.row_bytes);
    const int shift = chunk_shift(g.row_bytes);
    // The row this lane's pair scores: a round holds at most rounds_cap rows, so pairs past it
    // re-read the last row (their results are masked) instead of reading past the buffer.
    const unsigned char* const my_row =
        rows + static_cast<std::uint32_t>(min(lane & 15, rounds_cap - 1)) * stride_s;
    const int half = lane >> 4;

    // Launch statistics, per warp in 32 bits (a warp's counts stay far below 2^32; the byte
    // counters are derived from them when flushed): expansions, layer-0 / upper-layer distance
    // evaluations, link-block words read, re-rank rows, duplicates, prefetch hits, queries,
    // learned stops.
    std::uint32_t c_exp = 0, c_d0 = 0, c_du = 0, c_lw = 0, c_rr = 0, c_dup = 0, c_pf = 0, c_q = 0,
                  c_stop = 0;

    for (;;) {
        std::uint32_t qi = 0;
        if (lane == 0) {
            qi = atomicAdd(pass == 2 ? a.claim + 1 : a.claim, 1u);
        }
        qi = __shfl_sync(kFull, qi, 0);
        if (qi >= nq) {
            break;
        }
        if (pass == 2) {
            qi = a.order[qi];
            if (a.entry_ids[qi] == kNoId) {
                continue;  // failed its checks in the descent pass, which wrote its row
            }
        } else if (pass == 1 && lane == 0) {
            a.entry_ids[qi] = kNoId;  // until the descent below completes
        }
        const std::uint32_t k = a.k_per_q != nullptr ? a.k_per_q[qi] : a.k;
        std::uint32_t efq = a.ef_per_q != nullptr ? a.ef_per_q[qi] : a.ef;
        efq = efq > k ? efq : k;
        efq = efq < g.n ? efq : g.n;  // exhaustive beyond n: same result (no eviction possible)
        std::uint32_t* oid = a.out_ids + static_cast<std::size_t>(qi) * a.out_stride;
        float* od = a.out_dists + static_cast<std::size_t>(qi) * a.out_stride;
        if (efq > a.efcap) {
            if (lane == 0) {
                report(a.status, kErrCapacity, qi);
                a.out_counts[qi] = 0;
            }
            continue;
        }
        const int ef = static_cast<int>(efq);

        // 1. Query: load, check, normalize.
        const float* src = a.queries + static_cast<std::size_t>(qi) * a.qstride;
        bool bad = false;
        for (std::uint32_t e = lane; e < g.dim; e += 32) {
            const float v = src[e];
            bad |= !isfinite(v);
            q[e] = v;
        }
        __syncwarp();
        if (__any_sync(kFull, bad)) {
            if (lane == 0) {
                report(a.status, kErrNonFinite, qi);
                a.out_counts[qi] = 0;
            }
            for (std::uint32_t i = lane; i < a.out_stride; i += 32) {
                oid[i] = kNoId;
                od[i] = INFINITY;
            }
            continue;
        }
        if (g.metric == 2) {
            const float raw = warp_raw<kFP32, false>(q, reinterpret_cast<const unsigned char*>(q),
                                                     g.dim, g.row32 * 4, lane);
            const float n = sqrtf(raw);
            if (!(n > 0.0F) || !isfinite(n)) {
                if (lane == 0) {
                    report(a.status, kErrZeroCosine, qi);
                    a.out_counts[qi] = 0;
                }
                for (std::uint32_t i = lane; i < a.out_stride; i += 32) {
                    oid[i] = kNoId;
                    od[i] = INFINITY;
                }
                continue;
            }
            __syncwarp();
            for (std::uint32_t e = lane; e < g.dim; e += 32) {
                q[e] = __fdiv_rn(q[e], n);
            }
            __syncwarp();
        }
        if (pass != 2) {
            ++c_q;
        }
        if ((learned || tracing) && pass != 1) {
            // The constant features go to shared memory: the walk keeps no registers for them.
            const float qlen = sqrtf(warp_raw<kFP32, false>(
                q, reinterpret_cast<const unsigned char*>(q), g.dim, g.row32 * 4, lane));
            const float inv = 1.0F / fmaxf(qlen, 1e-20F);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float pr = inv * warp_raw<kFP32, false>(
                                           q, reinterpret_cast<const unsigned char*>(a.stop.proj + i * g.row32),
                                           g.dim, g.row32 * 4, lane);
                if (lane == 0) {
                    fc[2 + i] = pr;
                }
            }
            if (lane == 0) {
                fc[0] = qlen;
            }
        }
        std::uint32_t trace_points = 0;

        // 2. Entry point and greedy descent (in the layer-0 pass of an ordered launch, the
        // descent pass's result).
        std::uint32_t cur = g.entry;
        float curd = 0.0F;
        if (pass == 2) {
            cur = a.entry_ids[qi];
            curd = a.entry_d[qi];
        } else {
            // With the upper copy (the descent's blocks with each link's upper index, and the
            // rows of upper-layer nodes in one L2-resident allocation) the walk reads nothing
            // else; without it, the graph's own arrays. Same rows, same results.
            const bool compact = g.upper_aug != nullptr;
            const unsigned char* const up_rows = compact ? g.upper_rows : vecs;
            if (lane == 0) {
                fresh[0] = compact ? g.entry_ua : cur;
            }
            __syncwarp();
            gather_rows<true>(rows, stride_s, up_rows, fresh, 1, g.row_bytes, shift, lane);
            cp_async_wait<0>();
            __syncwarp();
            curd = lane_distance<P, kL2>(q, rows, g.dim, g.row_bytes);
            ++c_du;
            // cur's first upper block; a move takes the new node's from the candidates' indices,
            // which come with the block (upper copy) or are loaded while their rows are gathered.
            std::uint32_t cur_ua = g.max_level > 0 ? (compact ? g.entry_ua : g.upper_at[cur]) : 0;
            // The candidates' upper indices sit after the ids in `fresh` (it holds 2M >= 2 cap_up).
            std::uint32_t* const fresh_ua = fresh + g.cap_up;
            for (int layer = static_cast<int>(g.max_level); layer >= 1; --layer) {
                for (std::uint32_t hop = 0; hop <= g.n; ++hop) {
                    const std::uint32_t* block =
                        compact ? g.upper_aug + static_cast<std::size_t>(cur_ua + layer - 1) * (2 * g.stride_up)
                                : g.links_up + static_cast<std::size_t>(cur_ua + layer - 1) * g.stride_up;
                    int f = 0;
                    for (std::uint32_t c0 = 0; c0 < g.cap_up; c0 += 32) {
                        const std::uint32_t j = c0 + lane;
                        std::uint32_t id = j < g.cap_up ? block[j] : kNoId;
                        if (id != kNoId && id >= g.n) {
                            report(a.status, kErrBounds, qi);
                            id = kNoId;
                        }
                        const bool valid = id != kNoId;
                        const std::uint32_t m = __ballot_sync(kFull, valid);
                        if (valid) {
                            const int at = f + __popc(m & ((1u << lane) - 1u));
                            fresh[at] = id;
                            if (compact) {
                                fresh_ua[at] = block[g.stride_up + j];
                            }
                        }
                        f += __popc(m);
                    }
                    __syncwarp();
                    c_lw += 1 + f;
                    float best_d = INFINITY;
                    int best_i = 0x7FFFFFFF;
                    std::uint32_t best_ua = 0;
                    for (int s0 = 0; s0 < f; s0 += rounds_cap) {
                        const int cnt = min(rounds_cap, f - s0);
                        gather_rows<true>(rows, stride_s, up_rows, (compact ? fresh_ua : fresh) + s0, cnt,
                                          g.row_bytes, shift, lane);
                        // Candidates sit on this layer, so each has upper blocks (ids < n: checked).
                        const std::uint32_t ua =
                            lane < cnt ? (compact ? fresh_ua[s0 + lane] : g.upper_at[fresh[s0 + lane]]) : 0u;
                        cp_async_wait<0>();
                        __syncwarp();
                        const float pd = round_distance<P, kL2>(q, rows, stride_s, my_row, g.dim,
                                                                g.row_bytes, half, lane, cnt, rounds_cap);
                        float d = INFINITY;
                        int idx = 0x7FFFFFFF;
                        if (lane < cnt) {
                            d = pd;
                            idx = s0 + lane;
                        }
                        // The first strict minimum in link order: smallest (distance, position).
                        {
                            std::uint32_t bidx;
                            warp_argmin(d, static_cast<std::uint32_t>(idx), d, bidx);
                            idx = static_cast<int>(bidx);
                        }
                        const std::uint32_t round_ua = __shfl_sync(kFull, ua, (idx - s0) & 31);
                        if (d < best_d) {
                            best_d = d;
                            best_i = idx;
                            best_ua = round_ua;
                        }
                        __syncwarp();
                    }
                    c_du += f;
                    if (f > 0 && best_d < curd) {
                        cur = fresh[best_i];
                        cur_ua = best_ua;
                        curd = best_d;
                        __syncwarp();
                    } else {
                        break;
                    }
                }
            }
            if (pass == 1) {
                __syncwarp();
                if (lane == 0) {
                    a.entry_d[qi] = curd;
                    a.entry_ids[qi] = cur;
                }
                continue;
            }
        }

        // 3. Layer-0 beam.
        std::uint32_t epoch = 0;
        if (gtable != nullptr) {
            if (lane == 0) {
                epoch = a.gepoch[gwarp] + 1;
                a.gepoch[gwarp] = epoch;
            }
            epoch = __shfl_sync(kFull, epoch, 0);
            if (epoch == 0xFFFFFFFFu) {
                // Epochs wrapped (after 2^32 queries on this warp): clear and restart at 1.
                for (std::uint32_t i = lane; i < a.gstride; i += 32) {
                    gtable[i] = 0;
                }
                __syncwarp();
                epoch = 1;
                if (lane == 0) {
                    a.gepoch[gwarp] = 1;
                }
            }
        } else {
            for (std::uint32_t i = lane; i < a.hash_slots; i += 32) {
                table[i] = kNoId;
            }
        }
        __syncwarp();
        if (lane == 0) {
            visit(cur, epoch);
            rd[0] = curd;
            rid[0] = cur;
        }
        __syncwarp();
        RegBeam rb{};
        if constexpr (kRegR) {
            reg_beam_init(rb, curd, cur, lane);
        }
        int r = 1;
        int scan = 0;
        int slot = 0;
        std::uint32_t prefetched = kNoId;
        // kSpec (register beam over FP32 rows, plain search): each expansion also copies the link
        // block of R's first unexpanded entry after it (`spec`) into the other slot while it
        // runs. When the predicted next expansion is that entry (no candidate of this expansion
        // is closer), the next expansion is exactly it, so its visited filter and first row
        // gather run before this expansion's merge and the rows land while the merge runs
        // (`pre`: the filter and the first round's gather of the step were done by the previous
        // step; `f_pre` its fresh count). The filter's marks are the ones that expansion would
        // make, in the same order, so the walk is the same. Timed side by side on the 1M x 128
        // workload: FP32 ef 35 / 64 0.9 % / 2.2 % faster; the 96-register BF16 kernel spilled
        // more and was 1.6 % slower at ef 35, so it keeps the plain order.
        constexpr bool kSpec = kRegR && kLearn == kLearnNone && P == kFP32;
        bool pre = false;
        int f_pre = 0;
        if ((learned || tracing) && lane == 0) {
            fc[1] = curd;  // the layer-0 entry distance
        }
        int hops = 0;
        int last_change = 0;  // learned stop / traces: the expansion that last changed d_k
        for (std::uint32_t step = 0; step <= g.n; ++step) {
            int p;
            std::uint32_t node;
            if constexpr (kRegR) {
                p = reg_first_unexpanded(rb, scan, r, lane);
                if (p >= r) {
                    break;
                }
                node = reg_id(rb, p) & kIdMask;
                reg_mark_expanded(rb, p, lane);
            } else {
                p = first_unexpanded(rid, scan, r, lane);
                if (p >= r) {
                    break;
                }
                node = rid[p] & kIdMask;
            }
            __syncwarp();
            if (lane == 0) {
                rid[p] = node | kExpanded;
            }
            scan = p + 1;
            ++c_exp;
            // The previous step's prefetch (if any) lands in this step's slot: finish it first,
            // whether it is the block needed now or is about to be overwritten. (After a `pre`
            // step the links were read already and the first round's rows are in flight.)
            const bool pre_now = kSpec && pre;
            pre = false;
            std::uint32_t* links = lbuf + slot * g.stride0;
            if (!pre_now) {
                cp_async_wait<0>();
                __syncwarp();
                if (prefetched != node) {
                    const std::uint32_t* src_links = g.links0 + static_cast<std::size_t>(node) * g.stride0;
                    for (std::uint32_t x = lane; x < (g.stride0 >> 2); x += 32) {
                        cp_async16(links + 4 * x, src_links + 4 * x);
                    }
                    cp_async_commit();
                    cp_async_wait<0>();
                } else {
                    ++c_pf;
                }
                __syncwarp();
            } else {
                ++c_pf;
            }
            prefetched = kNoId;
            // Copies the links of `nxt` into the other slot (which holds no copy in flight).
            const auto copy_links = [&](std::uint32_t nxt) {
                std::uint32_t* other = lbuf + (slot ^ 1) * g.stride0;
                const std::uint32_t* src_links = g.links0 + static_cast<std::size_t>(nxt) * g.stride0;
                for (std::uint32_t x = lane; x < (g.stride0 >> 2); x += 32) {
                    cp_async16(other + 4 * x, src_links + 4 * x);
                }
            };
            // Starts copying the links of `nxt` (the predicted next expansion) into the other
            // slot; the copy lands while the current candidates are merged.
            const auto prefetch_links = [&](std::uint32_t nxt) {
                prefetched = nxt;
                if (nxt != kNoId) {
                    copy_links(nxt);
                    cp_async_commit();
                }
            };
            // The speculative copy: always one committed group (empty without an entry), so the
            // first round of a `pre` step can wait for everything but it.
            std::uint32_t spec = kNoId;
            if constexpr (kSpec) {
                const int pu = reg_first_unexpanded(rb, scan, r, lane);
                const std::uint32_t ui = reg_id(rb, pu < r ? pu : 0) & kIdMask;
                spec = pu < r ? ui : kNoId;
                if (spec != kNoId) {
                    copy_links(spec);
                }
                cp_async_commit();
            }
            // Unvisited neighbors of the block `lk`, in link order, into fresh[0, f); `count`
            // links present.
            const auto filter_links = [&](const std::uint32_t* lk, int& f, int& count) {
                f = 0;
                count = 0;
                for (std::uint32_t c0 = 0; c0 < g.cap0; c0 += 32) {
                    const std::uint32_t j = c0 + lane;
                    std::uint32_t id = j < g.cap0 ? lk[j] : kNoId;
                    if (id != kNoId && id >= g.n) {
                        report(a.status, kErrBounds, qi);
                        id = kNoId;
                    }
                    const bool present = id != kNoId;
                    count += __popc(__ballot_sync(kFull, present));
                    const bool isnew = present && visit(id, epoch);
                    const std::uint32_t m = __ballot_sync(kFull, isnew);
                    if (isnew) {
                        fresh[f + __popc(m & ((1u << lane) - 1u))] = id;
                    }
                    f += __popc(m);
                }
                __syncwarp();
                c_lw += 1 + count;
            };
            int f = 0;
            if (pre_now) {
                f = f_pre;  // filtered by the previous step (its link words counted there)
            } else {
                int count = 0;
                filter_links(links, f, count);
            }
            int kept_low = 0x7FFFFFFF;  // the lowest position a candidate was kept at
            for (int s0 = 0; s0 < f; s0 += rounds_cap) {
                const int cnt = min(rounds_cap, f - s0);
                if (pre_now && s0 == 0) {
                    cp_async_wait<1>();  // the rows; the newer group is the speculative copy
                } else {
                    gather_rows(rows, stride_s, vecs, fresh + s0, cnt, g.row_bytes, shift, lane);
                    cp_async_wait<0>();
                }
                __syncwarp();
                const bool valid = lane < cnt;
                const float pd = round_distance<P, kL2>(q, rows, stride_s, my_row, g.dim, g.row_bytes,
                                                        half, lane, cnt, rounds_cap);
                const float my_d = valid ? pd : INFINITY;
                const std::uint32_t my_id = valid ? fresh[s0 + lane] : kNoId;
                c_d0 += cnt;
                __syncwarp();
                if (s0 + rounds_cap >= f) {
                    // Last round: the next expansion is the closer of R's first unexpanded entry
                    // and this round's best candidate (when the merge will admit it). Exact except
                    // when that candidate duplicates an expanded entry (a visited-filter miss);
                    // then the next step fetches its links itself. When it is R's entry, it is
                    // exact without exception: every candidate the merge keeps is farther.
                    float bd;
                    std::uint32_t bi;
                    warp_argmin(my_d, my_id, bd, bi);
                    std::uint32_t nxt;
                    if constexpr (kRegR) {
                        const float wd = reg_d(rb, r - 1);
                        const std::uint32_t wi = reg_id(rb, r - 1) & kIdMask;
                        const bool admissible = bi != kNoId && (r < ef || closer(bd, bi, wd, wi));
                        const int pu = reg_first_unexpanded(rb, scan, r, lane);
                        nxt = admissible ? bi : kNoId;
                        const int pq = pu < r ? pu : 0;
                        const float ud = reg_d(rb, pq);
                        const std::uint32_t ui = reg_id(rb, pq) & kIdMask;
                        if (pu < r && (!admissible || closer(ud, ui, bd, bi))) {
                            nxt = ui;
                        }
                    } else {
                        const bool admissible =
                            bi != kNoId && (r < ef || closer(bd, bi, rd[r - 1], rid[r - 1] & kIdMask));
                        const int pu = first_unexpanded(rid, scan, r, lane);
                        nxt = admissible ? bi : kNoId;
                        if (pu < r) {
                            const std::uint32_t ui = rid[pu] & kIdMask;
                            if (!admissible || closer(rd[pu], ui, bd, bi)) {
                                nxt = ui;
                            }
                        }
                    }
                    __syncwarp();
                    if constexpr (kSpec) {
                        cp_async_wait<0>();  // the speculative copy (nothing else is in flight)
                        __syncwarp();
                        if (nxt != kNoId && nxt == spec) {
                            // The next expansion's filter and first row round, before the merge.
                            // This round's ids are in registers, so `fresh` is free.
                            int fn = 0;
                            int cn = 0;
                            filter_links(lbuf + (slot ^ 1) * g.stride0, fn, cn);
                            gather_rows(rows, stride_s, vecs, fresh, min(rounds_cap, fn), g.row_bytes,
                                        shift, lane);
                            f_pre = fn;
                            pre = true;
                            prefetched = nxt;
                        } else {
                            prefetch_links(nxt);
                        }
                    } else {
                        prefetch_links(nxt);
                    }
                }
                int low;
                if constexpr (kRegR) {
                    low = reg_merge_round(rb, rd, rid, r, ef, my_d, my_id, valid, lane, c_dup);
                } else {
                    low = merge_round(rd, rid, r, ef, my_d, my_id, valid, ap, lane, c_dup);
                }
                scan = min(scan, low);
                if constexpr (kLearn != kLearnNone) {
                    kept_low = min(kept_low, low);
                }
            }
            if (f == 0) {
                // Nothing scored: the next expansion is R's first unexpanded entry.
                if constexpr (kRegR) {
                    const int pu = reg_first_unexpanded(rb, scan, r, lane);
                    const std::uint32_t ui = reg_id(rb, pu < r ? pu : 0) & kIdMask;
                    const std::uint32_t nxt = pu < r ? ui : kNoId;
                    if (kSpec && nxt != kNoId && nxt == spec) {
                        prefetched = nxt;  // the speculative copy (the next step waits for it)
                    } else {
                        if constexpr (kSpec) {
                            cp_async_wait<0>();  // the speculative copy lands before the slot is reused
                            __syncwarp();
                        }
                        prefetch_links(nxt);
                    }
                } else {
                    const int pu = first_unexpanded(rid, scan, r, lane);
                    prefetch_links(pu < r ? rid[pu] & kIdMask : kNoId);
                }
            }
            slot ^= 1;
            ++hops;
            if (learned || tracing) {
                const int kk = r < static_cast<int>(k) ? r : static_cast<int>(k);
                // d_k changed when a candidate was kept above it (the merge's lowest kept
                // position); its value is sampled into the ring after every 4th expansion.
                if (kept_low < kk) {
                    last_change = hops;
                }
                if ((hops & 3) == 0) {
                    if (lane == 0) {
                        hist[(hops >> 2) & 7] = rd[kk - 1];
                    }
                    __syncwarp();
                }
                const int unchanged = hops - last_change;
                // Every 8 expansions: traces record the state; the stop consults the network
                // once the k-th distance has been unchanged for stop_gate expansions in a row
                // (0: at every checkpoint). While it still improves, the beam is not done.
                if (kLearn == kLearnStop) {
                    if ((hops & 7) == 0 && hops >= static_cast<int>(a.stop_min_hops) &&
                        r >= static_cast<int>(k) && static_cast<std::uint32_t>(unchanged) >= a.stop_gate &&
                        stop_decision(a.stop, fc, rd, r, static_cast<int>(k), hist, hops, unchanged, h1,
                                      a.stop_threshold, lane)) {
                        ++c_stop;
                        break;
                    }
                } else if ((hops & 7) == 0 &&
                    (tracing || static_cast<std::uint32_t>(unchanged) >= a.stop_gate)) {
                    float f[kFeatures];
                    stop_features(f, fc, rd, r, static_cast<int>(k), hist, hops, unchanged);
                    if (tracing && trace_points < a.trace.max_points) {
                        const std::size_t at = static_cast<std::size_t>(qi) * a.trace.max_points + trace_points;
                        if (lane < kFeatures) {
                            float v = f[0];
#pragma unroll
                            for (int c = 1; c < kFeatures; ++c) {
                                v = lane == c ? f[c] : v;
                            }
                            a.trace.features[at * kFeatures + lane] = v;
                        }
                        const std::uint32_t my = lane < kk ? (rid[lane] & kIdMask) : kNoId;
                        bool hit = false;
                        for (std::uint32_t t = 0; t < a.trace.truth_k; ++t) {
                            hit |= my == a.trace.truth[static_cast<std::size_t>(qi) * a.trace.truth_k + t];
                        }
                        const int hits = __popc(__ballot_sync(kFull, hit && my != kNoId));
                        if (lane == 0) {
                            a.trace.hits[at] = static_cast<std::uint8_t>(hits);
                        }
                        ++trace_points;
                    }
                    if (learned && hops >= static_cast<int>(a.stop_min_hops) && r >= static_cast<int>(k)) {
                        const float pr = stop_probability(a.stop, f, h1, lane);
                        if (pr >= a.stop_threshold) {
                            ++c_stop;
                            break;
                        }
                    }
                }
            }
        }
        cp_async_wait<0>();  // a prefetch may still be in flight
        __syncwarp();

        // Optional exact FP32 re-rank of the best candidates (low-precision traversal).
        const std::uint32_t rerank_n = a.rerank_per_k != 0 ? a.rerank_per_k * k : a.rerank;
        if (rerank_n > 0 && P != kFP32) {
            const int m = min(r, static_cast<int>(rerank_n));
            for (int i = lane; i < m; i += 32) {
                fresh[i] = rid[i] & kIdMask;
            }
            __syncwarp();
            const std::uint32_t row32b = g.row32 * 4;
            const std::uint32_t stride32 = padded_row_stride(row32b);
            const int shift32 = chunk_shift(row32b);
            // The walk is over: the visited filter, the link buffers and the row buffer form one
            // free region [off_hash, off_fresh) (at least one FP32 row: the row area is sized for
            // it). Two lanes score each row, so a round holds at most 16.
            unsigned char* const rrows = ws + a.off_hash;
            const int per_round =
                max(1, min(16, static_cast<int>((a.off_fresh - a.off_hash) / stride32)));
            const unsigned char* const my_rrow =
                rrows + static_cast<std::uint32_t>(min(lane & 15, per_round - 1)) * stride32;
            int rr = 0;
            for (int s0 = 0; s0 < m; s0 += per_round) {
                const int cnt = min(per_round, m - s0);
                gather_rows(rrows, stride32, reinterpret_cast<const unsigned char*>(g.vectors32),
                            fresh + s0, cnt, row32b, shift32, lane);
                cp_async_wait<0>();
                __syncwarp();
                const bool valid = lane < cnt;
                const float pd = row_distance<kFP32, kL2>(q, my_rrow, g.dim, row32b, half);
                const float my_d = valid ? pd : INFINITY;
                const std::uint32_t my_id = valid ? fresh[s0 + lane] : kNoId;
                c_rr += cnt;
                __syncwarp();
                // Build the re-ranked list in R's storage from scratch: the candidates' ids are
                // safe in `fresh`.
                if (s0 == 0) {
                    rr = 0;
                }
                unsigned long long unused = 0;
                merge_round(rd, rid, rr, static_cast<int>(k), my_d, my_id, valid, ap, lane, unused);
            }
            r = rr;
        }

        // 4. Results (a per-query k beyond the row width is cut to the width, so the count
        // never names entries that were not written).
        const int cnt = min(min(r, static_cast<int>(k)), static_cast<int>(a.out_stride));
        for (std::uint32_t i = lane; i < a.out_stride; i += 32) {
            if (static_cast<int>(i) < cnt) {
                oid[i] = rid[i] & kIdMask;
                od[i] = rd[i];
            } else {
                oid[i] = kNoId;
                od[i] = INFINITY;
            }
        }
        if (lane == 0) {
            a.out_counts[qi] = static_cast<std::uint32_t>(cnt);
        }
        if (tracing) {
            const std::uint32_t my = lane < cnt ? (rid[lane] & kIdMask) : kNoId;
            bool hit = false;
            for (std::uint32_t t = 0; t < a.trace.truth_k; ++t) {
                hit |= my == a.trace.truth[static_cast<std::size_t>(qi) * a.trace.truth_k + t];
            }
            const int hits = __popc(__ballot_sync(kFull, hit && my != kNoId));
            if (lane == 0) {
                a.trace.final_hits[qi] = static_cast<std::uint8_t>(hits);
                a.trace.points[qi] = trace_points;
            }
        }
        __syncwarp();
    }

    if (a.stats != nullptr && lane == 0) {
        using u64 = unsigned long long;
        atomicAdd(a.stats + kStatQueries, static_cast<u64>(c_q));
        atomicAdd(a.stats + kStatExpansions, static_cast<u64>(c_exp));
        atomicAdd(a.stats + kStatDist0, static_cast<u64>(c_d0));
        atomicAdd(a.stats + kStatDistUpper, static_cast<u64>(c_du));
        atomicAdd(a.stats + kStatLinkBytes, 4ull * c_lw);
        atomicAdd(a.stats + kStatRowBytes, (static_cast<u64>(c_d0) + c_du) * g.row_bytes);
        atomicAdd(a.stats + kStatRerankBytes, static_cast<u64>(c_rr) * (g.row32 * 4));
        atomicAdd(a.stats + kStatDuplicates, static_cast<u64>(c_dup));
        atomicAdd(a.stats + kStatPrefetchHits, static_cast<u64>(c_pf));
        atomicAdd(a.stats + kStatLearnedStops, static_cast<u64>(c_stop));
    }
}

std::uint32_t round_up(std::uint32_t x, std::uint32_t m) { return (x + m - 1) / m * m; }

// The claim order of an ordered launch's layer-0 pass: queries by their layer-0 entry distance,
// farthest first (the cost of a query's layer-0 walk grows with it), by a counting sort on the
// top 12 bits of the distance's order-preserving integer image (buckets a factor of ~1.09
// wide; order within a bucket is arbitrary). Queries that failed their checks go last. One
// block: the histogram and its scan live in shared memory.
constexpr int kOrderBuckets = 4096;
constexpr int kOrderThreads = 1024;

__device__ __forceinline__ std::uint32_t order_bucket(const SearchArgs& a, std::uint32_t i) {
    if (a.entry_ids[i] == kNoId) {
        return kOrderBuckets - 1;
    }
    std::uint32_t u = __float_as_uint(a.entry_d[i]);
    u = (u & 0x80000000u) != 0 ? ~u : (u | 0x80000000u);
    const std::uint32_t b = (kOrderBuckets - 1) - (u >> 20);
    return b < kOrderBuckets - 2 ? b : kOrderBuckets - 2;
}

__global__ void __launch_bounds__(kOrderThreads) order_kernel(const SearchArgs a) {
    // A programmatic dependent of the descent pass: the layer-0 pass may launch now; this kernel
    // waits in hardware until the descent has completed and its entries are visible.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    __shared__ std::uint32_t count[kOrderBuckets];
    __shared__ std::uint32_t warp_sum[kOrderThreads / 32];
    const std::uint32_t nq = a.nq_device != nullptr ? min(*a.nq_device, a.nq) : a.nq;
    const int t = static_cast<int>(threadIdx.x);
    for (int b = t; b < kOrderBuckets; b += kOrderThreads) {
        count[b] = 0;
    }
    __syncthreads();
    for (std::uint32_t i = t; i < nq; i += kOrderThreads) {
        atomicAdd(count + order_bucket(a, i), 1u);
    }
    __syncthreads();
    // Exclusive scan: each thread owns four consecutive buckets.
    constexpr int kPer = kOrderBuckets / kOrderThreads;
    std::uint32_t own[kPer];
    std::uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        own[j] = count[t * kPer + j];
        sum += own[j];
    }
    const int lane = t & 31;
    std::uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const std::uint32_t v = __shfl_up_sync(kFull, incl, o);
        incl += lane >= o ? v : 0u;
    }
    if (lane == 31) {
        warp_sum[t >> 5] = incl;
    }
    __syncthreads();
    if (t < 32) {
        const std::uint32_t w = warp_sum[t];
        std::uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const std::uint32_t v = __shfl_up_sync(kFull, wi, o);
            wi += t >= o ? v : 0u;
        }
        warp_sum[t] = wi - w;
    }
    __syncthreads();
    std::uint32_t base = warp_sum[t >> 5] + incl - sum;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        count[t * kPer + j] = base;
        base += own[j];
    }
    __syncthreads();
    for (std::uint32_t i = t; i < nq; i += kOrderThreads) {
        a.order[atomicAdd(count + order_bucket(a, i), 1u)] = i;
    }
}

thread_local int g_last_kernels = 1;

// Host-side launch bookkeeping. The dynamic shared-memory limit of each kernel is a property of
// the device's context, shared by every host thread: it is only ever raised, under a process-wide
// lock, so no launch can lower it under another thread's larger launch (which then fails with
// "invalid argument"); each thread remembers the limits it has seen, which stay valid since they
// only grow. The resident blocks of each (kernel, device, block size, shared memory) shape are
// cached per thread. A repeated launch makes no attribute or occupancy query.
struct SmemLimit {
    const void* kernel;
    int device;
    std::size_t bytes;
};
struct Residency {
    const void* kernel;
    int device;
    int threads;
    std::size_t smem;
    int blocks;
};
std::mutex g_smem_mutex;
std::vector<SmemLimit> g_smem_limits;              // the limits set, process-wide
thread_local std::vector<SmemLimit> g_smem_seen;   // limits this thread knows are in place
thread_local std::vector<Residency> g_residency;


// Blocks of `threads` threads and `smem` bytes that the device holds at once (SMs x per SM).
cudaError_t resident_blocks(const void* kernel, int device, int threads, std::size_t smem, int& blocks) {
    for (const Residency& r : g_residency) {
        if (r.kernel == kernel && r.device == device && r.threads == threads && r.smem == smem) {
            blocks = r.blocks;
            return cudaSuccess;
        }
    }
    int sms = 0;
    cudaError_t err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (err != cudaSuccess) {
        return err;
    }
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (err != cudaSuccess) {
        return err;
    }
    blocks = sms * (per_sm > 0 ? per_sm : 1);
    if (g_residency.size() < 64) {
        g_residency.push_back({kernel, device, threads, smem, blocks});
    }
    return cudaSuccess;
}

// The kernel of pass `kPass` for these arguments (the learned-stop variant when the stop or
// tracing is on).
template <int P, bool kL2, bool kRegR, int kPass>
const void* pass_kernel(const SearchArgs& args) {
    if constexpr (kPass == 1) {
        return reinterpret_cast<const void*>(&search_kernel<P, kL2, kRegR, kLearnNone, 1>);  // no stop
    } else {
        if (args.trace.truth != nullptr) {
            return reinterpret_cast<const void*>(&search_kernel<P, kL2, kRegR, kLearnTrace, kPass>);
        }
        if (args.stop_enabled != nullptr) {
            return reinterpret_cast<const void*>(&search_kernel<P, kL2, kRegR, kLearnStop, kPass>);
        }
        return reinterpret_cast<const void*>(&search_kernel<P, kL2, kRegR, kLearnNone, kPass>);
    }
}

template <int P, bool kL2, bool kRegR>
cudaError_t launch_typed(SearchArgs& args, const SearchPlan& plan, std::size_t smem,
                         cudaStream_t stream) {
    if (plan.warps_per_block < 1 || plan.warps_per_block * 32 > kMaxThreads<P, kRegR>) {
        return cudaErrorInvalidValue;  // a plan beyond max_warps_per_block
    }
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) {
        return err;
    }
    const int threads = plan.warps_per_block * 32;
    const std::uint32_t nq = args.nq;
    const std::uint32_t needed = (nq + plan.warps_per_block - 1) / plan.warps_per_block;
    // Sets the kernel's shared-memory limit and finds its grid: as many blocks as reside (or the
    // plan's count), trimmed to the batch unless the batch size is read on the device.
    const auto prepare = [&](const void* kernel, int& blocks) -> cudaError_t {
        cudaError_t e = raise_smem_limit(kernel, device, smem);
        if (e != cudaSuccess) {
            return e;
        }
        blocks = plan.blocks;
        if (blocks <= 0) {
            e = resident_blocks(kernel, device, threads, smem, blocks);
            if (e != cudaSuccess) {
                return e;
            }
        }
        if (args.nq_device == nullptr && static_cast<std::uint32_t>(blocks) > needed) {
            blocks = static_cast<int>(needed > 0 ? needed : 1);
        }
        return cudaSuccess;
    };
    // One global visited table per warp of the layer-0 grid: the caller's buffer must hold them.
    const auto check_tables = [&](int blocks) -> cudaError_t {
        if (plan.global_slots > 0) {
            if (args.gvisited == nullptr || args.gepoch == nullptr ||
                args.gslots != plan.global_slots || args.gstride < args.gslots ||
                static_cast<std::uint64_t>(blocks) * plan.warps_per_block > args.gwarps) {
                return cudaErrorInvalidValue;
            }
        } else {
            args.gvisited = nullptr;
        }
        return cudaSuccess;
    };
    using Kernel = void (*)(SearchArgs);
    // A launch of a kernel that walks the upper layers carries the graph's L2 access-policy
    // window over the upper copy (persisting hits, everything else in it streaming).
    const auto launch_walk = [&](const void* kernel, int blocks) -> cudaError_t {
        if (args.g.l2_window == nullptr) {
            reinterpret_cast<Kernel>(const_cast<void*>(kernel))<<<blocks, threads, smem, stream>>>(args);
            return cudaGetLastError();
        }
        cudaLaunchAttribute attr[1] = {};
        attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[0].val.accessPolicyWindow.base_ptr = const_cast<void*>(args.g.l2_window);
        attr[0].val.accessPolicyWindow.num_bytes = args.g.l2_window_bytes;
        attr[0].val.accessPolicyWindow.hitRatio = args.g.l2_hit_ratio;
        attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(static_cast<unsigned>(blocks));
        cfg.blockDim = dim3(static_cast<unsigned>(threads));
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        void* params[] = {&args};
        return cudaLaunchKernelExC(&cfg, kernel, params);
    };
    if (args.entry_ids == nullptr || args.entry_d == nullptr || args.order == nullptr) {
        const void* k0 = pass_kernel<P, kL2, kRegR, 0>(args);
        int blocks = 0;
        if (err = prepare(k0, blocks); err != cudaSuccess) {
            return err;
        }
        if (err = check_tables(blocks); err != cudaSuccess) {
            return err;
        }
        args.pass = 0;
        g_last_kernels = 1;
        return launch_walk(k0, blocks);
    }
    const void* k1 = pass_kernel<P, kL2, kRegR, 1>(args);
    const void* k2 = pass_kernel<P, kL2, kRegR, 2>(args);
    int blocks1 = 0;
    int blocks2 = 0;
    if (err = prepare(k1, blocks1); err != cudaSuccess) {
        return err;
    }
    if (err = prepare(k2, blocks2); err != cudaSuccess) {
        return err;
    }
    if (err = check_tables(blocks2); err != cudaSuccess) {
        return err;
    }
    // order_kernel and the layer-0 pass as programmatic dependents of the kernel before each
    // (their launch overlaps its end; griddepcontrol.wait in each orders the memory).
    const auto launch_dependent = [&](const void* kernel, int blocks, int block_threads,
                                      std::size_t shared) -> cudaError_t {
        cudaLaunchAttribute attr[1] = {};
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(static_cast<unsigned>(blocks));
        cfg.blockDim = dim3(static_cast<unsigned>(block_threads));
        cfg.dynamicSmemBytes = shared;
        cfg.stream = stream;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        void* params[] = {&args};
        return cudaLaunchKernelExC(&cfg, kernel, params);
    };
    args.pass = 1;
    if (err = launch_walk(k1, blocks1); err != cudaSuccess) {
        return err;
    }
    if (err = launch_dependent(reinterpret_cast<const void*>(&order_kernel), 1, kOrderThreads, 0);
        err != cudaSuccess) {
        return err;
    }
    args.pass = 2;
    g_last_kernels = 3;
    return launch_dependent(k2, blocks2, threads, smem);
}

}  // namespace

cudaError_t raise_smem_limit(const void* kernel, int device, std::size_t smem) {
    for (const SmemLimit& l : g_smem_seen) {
        if (l.kernel == kernel && l.device == device && smem <= l.bytes) {
            return cudaSuccess;
        }
    }
    const std::scoped_lock lock(g_smem_mutex);
    SmemLimit* entry = nullptr;
    for (SmemLimit& l : g_smem_limits) {
        if (l.kernel == kernel && l.device == device) {
            entry = &l;
        }
    }
    if (entry == nullptr || smem > entry->bytes) {
        const cudaError_t err = cudaFuncSetAttribute(
            kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (err != cudaSuccess) {
            return err;
        }
        if (entry == nullptr) {
            g_smem_limits.push_back({kernel, device, smem});
            entry = &g_smem_limits.back();
        } else {
            entry->bytes = smem;
        }
    }
    const SmemLimit seen = *entry;
    for (SmemLimit& l : g_smem_seen) {
        if (l.kernel == kernel && l.device == device) {
            l.bytes = seen.bytes;
            return cudaSuccess;
        }
    }
    g_smem_seen.push_back(seen);
    return cudaSuccess;
}

std::size_t plan_search(SearchArgs& a, const SearchPlan& plan) {
    const DeviceGraphView& g = a.g;
    a.efcap = plan.efcap;
    a.hash_slots = plan.global_slots > 0 ? 0 : plan.hash_slots;
    a.rows_cap = plan.rows_cap;
    std::uint32_t off = round_up(g.dim, 4) * 4;  // query
    a.off_r = off;
    off += round_up(plan.efcap * 8, 16);
    a.off_hash = off;
    off += a.hash_slots * 4;
    a.off_links = off;
    off += 2 * g.stride0 * 4;
    a.off_rows = off;
    const std::uint32_t row_area = plan.rows_cap * padded_row_stride(g.row_bytes);
    const std::uint32_t row32_area = padded_row_stride(g.row32 * 4);
    off += round_up(row_area > row32_area ? row_area : row32_area, 16);
    a.off_fresh = off;
    const std::uint32_t fresh_n = g.cap0 > g.cap_up ? g.cap0 : g.cap_up;
    const std::uint32_t fresh_need = fresh_n > a.rerank ? fresh_n : a.rerank;
    off += round_up((fresh_need > 32 ? fresh_need : 32) * 4, 16);
    a.off_ap = off;
    off += 32 * 4;
    a.off_hist = off;
    if (a.stop_enabled != nullptr || a.trace.truth != nullptr) {
        // Only the learned stop and its traces read the history ring and network scratch; the
        // kernel takes both flags from these same arguments, so the layout always matches.
        off += (kHist + kHidden + 8) * 4;
    }
    a.warp_bytes = round_up(off, 16);
    return static_cast<std::size_t>(a.warp_bytes) * plan.warps_per_block;
}

int max_warps_per_block(const DeviceGraphView& g, std::uint32_t efcap) {
    return (efcap <= kRegBeamCap && g.precision != kFP32 ? kMaxThreads<kBF16, true>
                                                         : kMaxThreads<kFP32, false>) / 32;
}

SearchPlan default_plan(const DeviceGraphView& g, std::uint32_t max_ef, bool allow_global) {
    SearchPlan p;
    std::uint32_t cap = 32;
    while (cap < max_ef) {
        cap <<= 1;
    }
    p.efcap = cap;
    // 16 slots per result entry, at least 1024: on the 1M x 128 workload a query visits ~600
    // nodes at ef = 36 and ~3k at ef = 512. The small table costs some filter misses (rows scored
    // twice) but keeps a warp's layout small: with BF16 / FP8 rows 20 warps reside per SM, with
    // FP32 rows 16 instead of 12 with a 2048-slot table (and no learned-stop scratch), which
    // made FP32 at ef = 36 / 64 11.7 % / 7.2 % faster, timed side by side, results identical.
    std::uint32_t slots = 1024;
    while (slots < 16 * cap && slots < 32768) {
        slots <<= 1;
    }
    p.hash_slots = slots;
    if (allow_global && cap >= 512) {
        // A shared-memory table of 16 slots per result entry (32 KB and up) would leave a few
        // warps per SM; a global table of 32 slots per entry (load <= 0.5) costs an L2 round per
        // filter instead. Side by side on the 1M x 128 workload the two are within 2 % at
        // ef = 256 and 512 (the shared table slightly ahead), so the switch is at 512; the
        // batcher's autotuner tries both from capacity 256.
        p.global_slots = 32 * cap;
        slots = 0;
    }
    // Rows staged per round: 16 keeps the per-warp footprint small enough for 12+ resident
    // warps per SM with FP32 rows; expansions with more unvisited neighbors take two rounds.
    p.rows_cap = g.cap0 < 16 ? (g.cap0 > 0 ? g.cap0 : 1) : 16;
    const std::size_t per_warp = round_up(g.dim, 4) * 4 + cap * 8 + slots * 4 + 2 * g.stride0 * 4 +
                                 p.rows_cap * padded_row_stride(g.row_bytes) + 1024;
    p.warps_per_block = per_warp * 4 <= 200 * 1024 ? 4 : (per_warp * 2 <= 200 * 1024 ? 2 : 1);
    return p;
}

std::uint32_t search_warps(SearchArgs& args, const SearchPlan& plan) {
    if (plan.blocks > 0) {
        return static_cast<std::uint32_t>(plan.blocks * plan.warps_per_block);
    }
    const std::size_t smem = plan_search(args, plan);
    int device = 0;
    cudaGetDevice(&device);
    const int threads = plan.warps_per_block * 32;
    // The grid launch_typed will pick for this kernel (same cached bookkeeping).
    const auto grid_of = [&](const void* kernel) {
        int blocks = 0;
        if (raise_smem_limit(kernel, device, smem) != cudaSuccess ||
            resident_blocks(kernel, device, threads, smem, blocks) != cudaSuccess) {
            int sms = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            return sms;
        }
        return blocks;
    };
    const bool l2 = args.g.metric == 0;
    // The kernels that read global tables (the whole-search and layer-0 passes) as launch_search
    // will pick them (register-beam variants for small capacities, learned-stop variants when the
    // stop or tracing is on); the tables must cover the larger of their grids.
    const bool reg = plan.efcap <= kRegBeamCap;
    const auto pick = [&](auto p_tag, auto pass_tag) -> const void* {
        constexpr int P = decltype(p_tag)::value;
        constexpr int kPass = decltype(pass_tag)::value;
        if (reg) {
            return l2 ? pass_kernel<P, true, true, kPass>(args) : pass_kernel<P, false, true, kPass>(args);
        }
        return l2 ? pass_kernel<P, true, false, kPass>(args) : pass_kernel<P, false, false, kPass>(args);
    };
    const auto pick_pass = [&](auto pass_tag) -> const void* {
        return args.g.precision == 0   ? pick(std::integral_constant<int, kFP32>{}, pass_tag)
               : args.g.precision == 1 ? pick(std::integral_constant<int, kBF16>{}, pass_tag)
                                       : pick(std::integral_constant<int, kFP8>{}, pass_tag);
    };
    const int grid = std::max(grid_of(pick_pass(std::integral_constant<int, 0>{})),
                              grid_of(pick_pass(std::integral_constant<int, 2>{})));
    return static_cast<std::uint32_t>(grid * plan.warps_per_block);
}

std::size_t global_visited_bytes(std::uint32_t stride, std::uint32_t warps) {
    if (stride == 0) {
        return 0;
    }
    return static_cast<std::size_t>(round_up(warps * 4, 256)) + static_cast<std::size_t>(warps) * stride * 8;
}

void bind_global_visited(SearchArgs& args, const SearchPlan& plan, void* buffer, std::uint32_t stride,
                         std::uint32_t warps) {
    if (plan.global_slots == 0 || buffer == nullptr) {
        args.gvisited = nullptr;
        return;
    }
    auto* b = static_cast<unsigned char*>(buffer);
    args.gepoch = reinterpret_cast<std::uint32_t*>(b);
    args.gvisited = reinterpret_cast<unsigned long long*>(b + round_up(warps * 4, 256));
    args.gslots = plan.global_slots;
    args.gstride = stride;
    args.gwarps = warps;
}

cudaError_t launch_search(SearchArgs& args, const SearchPlan& plan, cudaStream_t stream) {
    const std::size_t smem = plan_search(args, plan);
    const bool l2 = args.g.metric == 0;
    if (plan.efcap <= kRegBeamCap) {
        switch (args.g.precision) {
            case 0:
                return l2 ? launch_typed<kFP32, true, true>(args, plan, smem, stream)
                          : launch_typed<kFP32, false, true>(args, plan, smem, stream);
            case 1:
                return l2 ? launch_typed<kBF16, true, true>(args, plan, smem, stream)
                          : launch_typed<kBF16, false, true>(args, plan, smem, stream);
            default:
                return l2 ? launch_typed<kFP8, true, true>(args, plan, smem, stream)
                          : launch_typed<kFP8, false, true>(args, plan, smem, stream);
        }
    }
    switch (args.g.precision) {
        case 0:
            return l2 ? launch_typed<kFP32, true, false>(args, plan, smem, stream)
                      : launch_typed<kFP32, false, false>(args, plan, smem, stream);
        case 1:
            return l2 ? launch_typed<kBF16, true, false>(args, plan, smem, stream)
                      : launch_typed<kBF16, false, false>(args, plan, smem, stream);
        default:
            return l2 ? launch_typed<kFP8, true, false>(args, plan, smem, stream)
                      : launch_typed<kFP8, false, false>(args, plan, smem, stream);
    }
}

int search_kernels_per_launch() { return g_last_kernels; }

}  // namespace vdx::dev
