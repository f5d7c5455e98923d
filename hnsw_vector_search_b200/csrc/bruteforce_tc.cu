// Exact brute force through the tensor cores (tcgen05 + TMEM + TMA), certified against the
// reference's FP32 results.
//
// 1. prep: each vector is split into bfloat16 hi = bf16(x) and lo = bf16(x - hi) (zero-padded to
//    a multiple of 64 components); squared norms in FP32. For integer data in [-256, 256] (the
//    SIFT-like workloads) lo is zero and every product and partial sum is exact in FP32.
// 2. score (bf_tc_kernel): a CTA owns 128 queries (the MMA's M) and streams a chunk of the
//    stored vectors through shared memory in tiles of 128 rows (N), K in 64-element swizzled
//    chunks. One thread issues TMA loads (no multicast), one thread issues
//    tcgen05.mma.kind::f16 (BF16 x BF16 -> FP32 in TMEM, the terms hi*hi + hi*lo + lo*hi when
//    the data needs them), and eight warps read the 128 x 128 FP32 tile out of TMEM (double
//    buffered, so the next tile's MMAs overlap), score it (2 q.x - ||x||^2, or q.x) and keep
//    each query's best `kc` candidates of the chunk in shared memory (one query per thread and
//    column half), starting from the best bound the query's other lists have published.
// 3. merge (bf_tc_merge_kernel): per query, the best `kc` candidates over all lists are
//    re-scored with the reference's exact FP32 order (lane_distance) and sorted by `closer`.
//    The query is certified when its k-th exact distance is below every excluded vector's
//    lowest possible exact distance (the smallest excluded approximate distance minus the
//    scoring error bound); for integer data the bound is exact arithmetic.
// 4. queries that are not certified are recomputed by the exact CUDA-core kernel.
// So the result is the reference's, ids and distance bits, for every query.
//
// Every mbarrier wait is bounded (1 s of %globaltimer); a timeout sets an error word, every role
// stops, outstanding copies and MMAs are waited for (again bounded), TMEM is freed, and the host
// raises an error. Nothing waits on another CTA.

#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "bruteforce.cuh"
#include "common.cuh"

namespace vdx::dev {
namespace {

constexpr int kBM = 128;                        // queries per tile (MMA M, TMEM lanes)
constexpr int kBN = 128;                        // stored rows per tile (MMA N, TMEM columns)
constexpr int kBK = 64;                         // K elements per 128-byte swizzled chunk
constexpr std::uint32_t kChunk = kBM * kBK * 2;  // 16 KB: one 128 x 64 bf16 chunk
constexpr int kThreads = 384;  // 4 role warps + up to 8 epilogue warps
constexpr std::uint64_t kWaitNs = 1000000000ull;
constexpr std::uint32_t kTmemCols = 2 * kBN;   // two accumulator buffers

// -------------------------------------------------------------------------------------------
// PTX wrappers

__device__ __forceinline__ std::uint64_t now_ns() {
    std::uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(std::uint32_t a, std::uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(std::uint32_t a, std::uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(std::uint32_t a) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_try(std::uint32_t a, std::uint32_t parity) {
    std::uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase with `parity` to complete; false after `limit_ns` or once another role
// has aborted. The pipeline's waits use the launch's limit (kWaitNs unless a test shortens it);
// the drains before the CTA exits always use the full kWaitNs.
__device__ __forceinline__ bool mbar_wait(std::uint32_t a, std::uint32_t parity,
                                          volatile std::uint32_t* abort_flag, std::uint64_t limit_ns) {
    if (mbar_try(a, parity)) {
        return true;
    }
    const std::uint64_t t0 = now_ns();
    for (;;) {
        if (mbar_try(a, parity)) {
            return true;
        }
        if (*abort_flag != 0 || now_ns() - t0 > limit_ns) {
            return false;
        }
    }
}
// Bounded by the full kWaitNs, for the drains: true when the phase completed.
__device__ __forceinline__ bool mbar_drain(std::uint32_t a, std::uint32_t parity) {
    const std::uint64_t t0 = now_ns();
    while (!mbar_try(a, parity)) {
        if (now_ns() - t0 > kWaitNs) {
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void tma_load_2d(std::uint32_t dst, const CUtensorMap* map, int x,
                                            int y, std::uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<std::uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Shared-memory matrix descriptor of a K-major tile written by TMA with 128-byte swizzling:
// rows of 128 bytes, 8-row atoms 1024 bytes apart (SBO), version 1, layout SWIZZLE_128B.
__device__ __forceinline__ std::uint64_t sw128_desc(std::uint32_t saddr) {
    return static_cast<std::uint64_t>((saddr & 0x3FFFFu) >> 4) | (std::uint64_t{1} << 16) |
           (std::uint64_t{1024 >> 4} << 32) | (std::uint64_t{1} << 46) | (std::uint64_t{2} << 61);
}
// Instruction descriptor: BF16 A and B, FP32 accumulator, both K-major, M = 128, N = 128.
constexpr std::uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                                 (static_cast<std::uint32_t>(kBN >> 3) << 17) |
                                 (static_cast<std::uint32_t>(kBM >> 4) << 24);
__device__ __forceinline__ void mma_bf16(std::uint32_t d_tmem, std::uint64_t a, std::uint64_t b,
                                         std::uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(std::uint32_t mbar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
        : "memory");
}
// The MMAs of one 128 x 128 tile: K in KC chunks of 64, 16 per MMA, the hi * hi products plus
// hi * lo (XLO) and lo * hi (QLO) when the data need them. Fully unrolled with compile-time
// offsets: issued from a loop with a run-time trip count and branches, each MMA took about three
// times as long to issue as the tensor core takes to run it (measured on a B200).
template <int KC, bool XLO, bool QLO>
__device__ __forceinline__ void mma_tile(std::uint32_t d_tmem, std::uint32_t a_hi, std::uint32_t a_lo,
                                         std::uint32_t bs) {
#pragma unroll
    for (int c = 0; c < KC; ++c) {
#pragma unroll
        for (int kk = 0; kk < kBK / 16; ++kk) {
            const std::uint32_t off = static_cast<std::uint32_t>(c) * kChunk + static_cast<std::uint32_t>(kk) * 32;
            const std::uint64_t ah = sw128_desc(a_hi + off);
            const std::uint64_t bh = sw128_desc(bs + off);
            mma_bf16(d_tmem, ah, bh, (c | kk) != 0 ? 1u : 0u);
            if (XLO) {
                mma_bf16(d_tmem, ah, sw128_desc(bs + KC * kChunk + off), 1u);
            }
            if (QLO) {
                mma_bf16(d_tmem, sw128_desc(a_lo + off), bh, 1u);
            }
        }
    }
}
template <int KC>
__device__ __forceinline__ void mma_tile_terms(bool xlo, bool qlo, std::uint32_t d_tmem, std::uint32_t a_hi,
                                               std::uint32_t a_lo, std::uint32_t bs) {
    if (xlo) {
        if (qlo) {
            mma_tile<KC, true, true>(d_tmem, a_hi, a_lo, bs);
        } else {
            mma_tile<KC, true, false>(d_tmem, a_hi, a_lo, bs);
        }
    } else if (qlo) {
        mma_tile<KC, false, true>(d_tmem, a_hi, a_lo, bs);
    } else {
        mma_tile<KC, false, false>(d_tmem, a_hi, a_lo, bs);
    }
}
// One tile's MMAs for kchunks in 1..4 (the plan admits no other count).
__device__ __forceinline__ void mma_tile_any(std::uint32_t kchunks, bool xlo, bool qlo, std::uint32_t d_tmem,
                                             std::uint32_t a_hi, std::uint32_t a_lo, std::uint32_t bs) {
    switch (kchunks) {
        case 1: mma_tile_terms<1>(xlo, qlo, d_tmem, a_hi, a_lo, bs); break;
        case 2: mma_tile_terms<2>(xlo, qlo, d_tmem, a_hi, a_lo, bs); break;
        case 3: mma_tile_terms<3>(xlo, qlo, d_tmem, a_hi, a_lo, bs); break;
        default: mma_tile_terms<4>(xlo, qlo, d_tmem, a_hi, a_lo, bs); break;
    }
}
__device__ __forceinline__ void tmem_ld32(std::uint32_t taddr, std::uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// d0 = fma(c, s0, b0), d1 = fma(c, s1, b1) in one paired instruction (each half rounded as a
// scalar fma).
__device__ __forceinline__ void fma2(float& d0, float& d1, float c, float s0, float s1, float b0,
                                     float b1) {
    std::uint64_t cc, ss, bb, dd;
    asm("mov.b64 %0, {%1, %1};" : "=l"(cc) : "f"(c));
    asm("mov.b64 %0, {%1, %2};" : "=l"(ss) : "f"(s0), "f"(s1));
    asm("mov.b64 %0, {%1, %2};" : "=l"(bb) : "f"(b0), "f"(b1));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(dd) : "l"(cc), "l"(ss), "l"(bb));
    asm("mov.b64 {%0, %1}, %2;" : "=f"(d0), "=f"(d1) : "l"(dd));
}
__device__ __forceinline__ float max3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
// 32 consecutive score offsets (one 32-column group), as eight broadcast 16-byte loads.
__device__ __forceinline__ void load_bias(float4 (&v)[8], const float* src) {
    const float4* s = reinterpret_cast<const float4*>(src);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        v[i] = __ldg(s + i);
    }
}

// Order-preserving map of floats to u32 (so atomicMax on the key is max on the float).
__device__ __forceinline__ std::uint32_t float_to_key(float f) {
    const std::uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
// Keys below that of -inf (0x007FFFFF) would be NaNs and are never produced: the zeroed array
// means "no floor yet" (-inf).
__device__ __forceinline__ float key_to_float(std::uint32_t k) {
    if (k < 0x007FFFFFu) {
        return -INFINITY;
    }
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// One score against a thread's candidate list (column e of [kc][128] arrays, best first, ties
// by the lower id). `thr` / `thr_i` is the acceptance bound (kNoId: ties with it are accepted);
// it only rises, to the list's kc-th once the list is full.
__device__ __forceinline__ void consider(float v, std::uint32_t id, float* list_d,
                                         std::uint32_t* list_i, std::uint32_t e, std::uint32_t kc,
                                         std::uint32_t& count, float& thr, std::uint32_t& thr_i) {
    if (!(v > thr || (v == thr && id < thr_i))) {
        return;
    }
    std::uint32_t pos = count < kc ? count : kc - 1;
    while (pos > 0) {
        const float pv = list_d[(pos - 1) * kBM + e];
        const std::uint32_t pi = list_i[(pos - 1) * kBM + e];
        if (!(v > pv || (v == pv && id < pi))) {
            break;
        }
        list_d[pos * kBM + e] = pv;
        list_i[pos * kBM + e] = pi;
        --pos;
    }
    list_d[pos * kBM + e] = v;
    list_i[pos * kBM + e] = id;
    if (count < kc) {
        ++count;
    }
    if (count == kc) {
        const float kth = list_d[(kc - 1) * kBM + e];
        const std::uint32_t kth_i = list_i[(kc - 1) * kBM + e];
        if (kth > thr || (kth == thr && thr_i == kNoId)) {
            thr = kth;
            thr_i = kth_i;
        }
    }
}

// -------------------------------------------------------------------------------------------
// Kernel parameters

// Work split: the stored rows' tpq tiles of 128 are cut into `nchunks` runs of equal length (to
// a tile); a work item is one (query tile, chunk) pair, item = chunk * qtiles + query tile, and
// CTA b takes items b, b + grid, b + 2 grid, ... So the CTAs of one wave stream the same one to
// three chunks side by side (a row tile is read from HBM about once per wave and then served by
// L2), and a query's chunks are taken in order, each list starting from the best bound that the
// query's other lists have published (`floor_key`).
__host__ __device__ inline std::uint32_t chunk_begin(std::uint32_t ch, std::uint32_t tpq,
                                                     std::uint32_t nchunks) {
    return static_cast<std::uint32_t>(static_cast<std::uint64_t>(ch) * tpq / nchunks);
}

struct TcParams {
    std::uint32_t nq, n, dim, kchunks, qtiles, nchunks, tpq, kc, stages, metric;
    std::uint32_t halves;                 // epilogue warps per TMEM lane quarter (column halves)
    std::uint32_t base_lo;                // the stored vectors have nonzero lo parts
    const std::uint32_t* query_flags;     // bit 0: some query has a nonzero lo part
    const float* qnorm;                   // [nq]
    const float* xnorm;                   // [n rounded up to a tile]: the score bias
    std::uint32_t* cand_ids;              // [nq][nchunks * halves][kc]
    float* cand_d;
    float* cand_tau;                      // [nq][nchunks * halves]
    std::uint32_t* floor_key;             // [nq] best kc-th score any list holds (ordered key)
    std::uint32_t* quarter_key;           // [nq][nchunks * halves] each list's (kc / 4)-th score
    std::uint32_t* error;                 // status word: 5 on a timeout
    std::uint64_t wait_ns;                // limit of each pipeline wait (the drains keep kWaitNs)
    std::uint32_t off_b, off_lists, off_bar;  // smem offsets from the 1024-aligned base
};

__global__ void __launch_bounds__(kThreads, 1)
    bf_tc_kernel(const __grid_constant__ CUtensorMap tq_hi, const __grid_constant__ CUtensorMap tq_lo,
                 const __grid_constant__ CUtensorMap tx_hi, const __grid_constant__ CUtensorMap tx_lo,
                 const TcParams p) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const std::uint32_t raw_addr = smem_addr(smem_raw);
    const std::uint32_t base_addr = (raw_addr + 1023u) & ~1023u;
    unsigned char* base = smem_raw + (base_addr - raw_addr);
    const int warp = static_cast<int>(threadIdx.x >> 5);
    const int lane = static_cast<int>(threadIdx.x & 31);

    const std::uint32_t S = p.stages;
    const bool qlo = (*p.query_flags & 1u) != 0;
    const bool xlo = p.base_lo != 0;
    const std::uint32_t a_hi = base_addr;
    const std::uint32_t a_lo = base_addr + p.kchunks * kChunk;
    const std::uint32_t stage_bytes = (xlo ? 2u : 1u) * p.kchunks * kChunk;
    const std::uint32_t b0 = base_addr + p.off_b;
    const std::uint32_t bar = base_addr + p.off_bar;
    const auto full = [&](std::uint32_t s) { return bar + 8 * s; };
    const auto empty = [&](std::uint32_t s) { return bar + 8 * (S + s); };
    const std::uint32_t a_full = bar + 8 * (2 * S);
    const std::uint32_t a_empty = a_full + 8;
    const std::uint32_t tfull0 = a_full + 16;   // two
    const std::uint32_t tempty0 = a_full + 32;  // two
    const std::uint32_t drain = a_full + 48;
    std::uint32_t* holder = reinterpret_cast<std::uint32_t*>(base + p.off_bar + 8 * (2 * S) + 56);
    volatile std::uint32_t* abort_flag = holder + 1;

    if (threadIdx.x == 0) {
        for (std::uint32_t s = 0; s < S; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        mbar_init(a_full, 1);
        mbar_init(a_empty, 1);
        mbar_init(tfull0, 1);
        mbar_init(tfull0 + 8, 1);
        mbar_init(tempty0, kBM * p.halves);
        mbar_init(tempty0 + 8, kBM * p.halves);
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(holder)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const std::uint32_t tmem = *holder;

    const std::uint32_t items = p.qtiles * p.nchunks;
    const auto fail = [&]() {
        *abort_flag = 1;
        atomicCAS(p.error, 0u, 5u);  // the host raises "device wait timed out"
    };

    if (warp == 0 && lane == 0) {
        // TMA producer.
        std::uint32_t it = 0, item_idx = 0, a_loads = 0;
        bool ok = true;
        for (std::uint32_t item = blockIdx.x; ok && item < items; item += gridDim.x, ++item_idx) {
            const std::uint32_t qt = item % p.qtiles;
            const std::uint32_t ch = item / p.qtiles;
            if (item_idx > 0 && !mbar_wait(a_empty, (item_idx - 1) & 1u, abort_flag, p.wait_ns)) {
                fail();
                ok = false;
                break;
            }
            mbar_expect_tx(a_full, (qlo ? 2u : 1u) * p.kchunks * kChunk);
            for (std::uint32_t c = 0; c < p.kchunks; ++c) {
                tma_load_2d(a_hi + c * kChunk, &tq_hi, static_cast<int>(c * kBK),
                            static_cast<int>(qt * kBM), a_full);
                if (qlo) {
                    tma_load_2d(a_lo + c * kChunk, &tq_lo, static_cast<int>(c * kBK),
                                static_cast<int>(qt * kBM), a_full);
                }
            }
            ++a_loads;
            const std::uint32_t t0 = chunk_begin(ch, p.tpq, p.nchunks);
            const std::uint32_t row0 = t0 * kBN;
            const std::uint32_t tiles = chunk_begin(ch + 1, p.tpq, p.nchunks) - t0;
            for (std::uint32_t t = 0; t < tiles; ++t, ++it) {
                const std::uint32_t s = it % S;
                const std::uint32_t ph = (it / S) & 1u;
                if (!mbar_wait(empty(s), ph ^ 1u, abort_flag, p.wait_ns)) {
                    fail();
                    ok = false;
                    break;
                }
                mbar_expect_tx(full(s), stage_bytes);
                const std::uint32_t bs = b0 + s * stage_bytes;
                const int y = static_cast<int>(row0 + t * kBN);
                for (std::uint32_t c = 0; c < p.kchunks; ++c) {
                    tma_load_2d(bs + c * kChunk, &tx_hi, static_cast<int>(c * kBK), y, full(s));
                    if (xlo) {
                        tma_load_2d(bs + (p.kchunks + c) * kChunk, &tx_lo, static_cast<int>(c * kBK),
                                    y, full(s));
                    }
                }
            }
        }
        // Every copy this thread issued lands before the CTA exits, whichever role stopped the
        // pipeline (bounded by the full kWaitNs): the loads of the last min(S, it) tiles, tile i
        // on stage i % S with phase parity (i / S) & 1, and the last query tile (phase
        // a_loads - 1 of a_full). On the normal path these phases are long complete and the
        // waits return at once.
        (void)ok;
        for (std::uint32_t i = it > S ? it - S : 0; i < it; ++i) {
            mbar_drain(full(i % S), (i / S) & 1u);
        }
        if (a_loads > 0) {
            mbar_drain(a_full, (a_loads - 1) & 1u);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer.
        std::uint32_t it = 0, acc_it = 0, item_idx = 0;
        bool ok = true;
        for (std::uint32_t item = blockIdx.x; ok && item < items; item += gridDim.x, ++item_idx) {
            const std::uint32_t ch = item / p.qtiles;
            const std::uint32_t t0 = chunk_begin(ch, p.tpq, p.nchunks);
            const std::uint32_t row0 = t0 * kBN;
            const std::uint32_t tiles = chunk_begin(ch + 1, p.tpq, p.nchunks) - t0;
            if (!mbar_wait(a_full, item_idx & 1u, abort_flag, p.wait_ns)) {
                fail();
                ok = false;
                break;
            }
            tc_fence_after();
            for (std::uint32_t t = 0; t < tiles; ++t, ++it, ++acc_it) {
                const std::uint32_t s = it % S;
                const std::uint32_t b = acc_it & 1u;
                if (!mbar_wait(tempty0 + 8 * b, ((acc_it >> 1) & 1u) ^ 1u, abort_flag, p.wait_ns) ||
                    !mbar_wait(full(s), (it / S) & 1u, abort_flag, p.wait_ns)) {
                    fail();
                    ok = false;
                    break;
                }
                tc_fence_after();
                mma_tile_any(p.kchunks, xlo, qlo, tmem + b * kBN, a_hi, a_lo, b0 + s * stage_bytes);
                mma_commit(empty(s));
                mma_commit(tfull0 + 8 * b);
            }
            if (ok) {
                mma_commit(a_empty);
            }
        }
        // Every MMA this thread issued has completed before TMEM is freed (bounded).
        mma_commit(drain);
        mbar_drain(drain, 0);
    } else if (warp >= 4 && static_cast<std::uint32_t>(warp - 4) < 4 * p.halves) {
        // Epilogue: thread e owns query row e of the tile (TMEM lane e) in column half `half`
        // of every tile (with halves = 2, two warps per TMEM lane quarter split the 128 columns,
        // so two warps per scheduler hide each other's latency), with its own candidate list per
        // item (the merge treats each half's list like a chunk of its own). It works in score
        // space, t = 2 q.x - ||x||^2 (L2) or t = q.x (inner product), larger is closer; the
        // per-row offset (-||x||^2, or -0; -inf for padding rows) is read 32 at a time with
        // broadcast 16-byte loads issued one group ahead, and a group of 32 scores enters the
        // insertion path only if its best score can beat the list's current bound.
        const std::uint32_t e = static_cast<std::uint32_t>((warp & 3) * 32 + lane);
        const std::uint32_t half = static_cast<std::uint32_t>(warp - 4) >> 2;
        const std::uint32_t groups = (kBN / 32) / p.halves;  // 32-column groups per half
        const std::uint32_t g0 = half * groups;
        const std::uint32_t lists = p.nchunks * p.halves;
        float* list_d = reinterpret_cast<float*>(base + p.off_lists + half * p.kc * kBM * 8);  // [kc][128]
        std::uint32_t* list_i = reinterpret_cast<std::uint32_t*>(base + p.off_lists + half * p.kc * kBM * 8 +
                                                                 p.kc * kBM * 4);
        const std::uint32_t lane_base = static_cast<std::uint32_t>((warp & 3) * 32) << 16;
        const bool l2 = p.metric == 0;
        const float c2 = l2 ? 2.0F : 1.0F;
        std::uint32_t acc_it = 0;
        bool ok = true;
        for (std::uint32_t item = blockIdx.x; ok && item < items; item += gridDim.x) {
            const std::uint32_t qt = item % p.qtiles;
            const std::uint32_t ch = item / p.qtiles;
            const std::uint32_t row = qt * kBM + e;
            const bool live = row < p.nq;
            const std::uint32_t t0 = chunk_begin(ch, p.tpq, p.nchunks);
            const std::uint32_t row0 = t0 * kBN;
            const std::uint32_t tiles = chunk_begin(ch + 1, p.tpq, p.nchunks) - t0;
            std::uint32_t count = 0;
            // Scores at or below `floor` cannot reach the global best kc: another list already
            // holds kc better ones (every list is part of the merge).
            float floor = live ? key_to_float(__ldcg(p.floor_key + row)) : INFINITY;
            float thr = floor;            // acceptance bound: the floor, then the list's kc-th
            std::uint32_t thr_i = kNoId;  // kNoId: ties with the bound are accepted
            float4 nb[8];
            load_bias(nb, p.xnorm + row0 + g0 * 32);
            for (std::uint32_t t = 0; t < tiles; ++t, ++acc_it) {
                const std::uint32_t b = acc_it & 1u;
                if (!mbar_wait(tfull0 + 8 * b, (acc_it >> 1) & 1u, abort_flag, p.wait_ns)) {
                    fail();
                    ok = false;
                    break;
                }
                tc_fence_after();
                for (std::uint32_t g = 0; g < groups; ++g) {
                    const std::uint32_t cc = g0 + g;
                    const std::uint32_t id0 = row0 + t * kBN + cc * 32;
                    // The offsets of the next group (this tile's next, or the next tile's first;
                    // the current group again after the item's last), in flight while this
                    // group's scores are read and scored.
                    const std::uint32_t nxt = g + 1 < groups ? id0 + 32
                                              : t + 1 < tiles ? row0 + (t + 1) * kBN + g0 * 32
                                                              : id0;
                    float4 nx[8];
                    load_bias(nx, p.xnorm + nxt);
                    std::uint32_t r[32];
                    tmem_ld32(tmem + lane_base + b * kBN + cc * 32, r);
                    if (g == groups - 1) {
                        tc_fence_before();
                        mbar_arrive(tempty0 + 8 * b);
                    }
                    // t = c * s + nb with c = 2 (L2) or 1 and nb = -||x||^2 (L2), -0 (inner
                    // product) or -inf (padding rows): two scores per f32x2 FMA, each rounded
                    // like a scalar fmaf. Everything stays in registers (static indices only).
                    float sc[32];
#pragma unroll
                    for (int q4 = 0; q4 < 8; ++q4) {
                        fma2(sc[4 * q4], sc[4 * q4 + 1], c2, __uint_as_float(r[4 * q4]),
                             __uint_as_float(r[4 * q4 + 1]), nb[q4].x, nb[q4].y);
                        fma2(sc[4 * q4 + 2], sc[4 * q4 + 3], c2, __uint_as_float(r[4 * q4 + 2]),
                             __uint_as_float(r[4 * q4 + 3]), nb[q4].z, nb[q4].w);
                    }
#pragma unroll
                    for (int q4 = 0; q4 < 8; ++q4) {
                        nb[q4] = nx[q4];
                    }
                    // Best of each triple, then of the 32, with three-input max; most groups
                    // stop here.
                    float m3[11];
#pragma unroll
                    for (int i = 0; i < 10; ++i) {
                        m3[i] = max3(sc[3 * i], sc[3 * i + 1], sc[3 * i + 2]);
                    }
                    m3[10] = fmaxf(sc[30], sc[31]);
                    const float mx = max3(max3(m3[0], m3[1], m3[2]), max3(m3[3], m3[4], m3[5]),
                                          max3(max3(m3[6], m3[7], m3[8]), m3[9], m3[10]));
                    if (!live || !(mx >= thr)) {
                        continue;
                    }
                    // Rare path, kept small (it runs cold, so its size costs instruction-cache
                    // misses): the triples whose best may qualify, in column order, each picked
                    // out of the registers by predicated moves, their scores offered to one copy
                    // of the insertion code. The bound only rises, so a triple that failed under
                    // an older bound stays out under a newer one.
                    std::uint32_t tm = 0;
#pragma unroll
                    for (int i = 0; i < 11; ++i) {
                        tm |= m3[i] >= thr ? 1u << i : 0u;
                    }
                    while (tm != 0) {
                        const int i = __ffs(static_cast<int>(tm)) - 1;
                        tm &= tm - 1;
                        float v0 = 0.0F, v1 = 0.0F, v2 = 0.0F;
#pragma unroll
                        for (int k = 0; k < 11; ++k) {
                            if (k == i) {
                                v0 = sc[3 * k];
                                v1 = sc[3 * k + 1];
                                v2 = k < 10 ? sc[3 * k + 2] : 0.0F;
                            }
                        }
                        const std::uint32_t idb = id0 + 3u * static_cast<std::uint32_t>(i);
                        const int width = i < 10 ? 3 : 2;
#pragma unroll 1
                        for (int jj = 0; jj < width; ++jj) {
                            consider(jj == 0 ? v0 : (jj == 1 ? v1 : v2), idb + static_cast<std::uint32_t>(jj),
                                     list_d, list_i, e, p.kc, count, thr, thr_i);
                        }
                    }
                }
                if (live && (t & 31u) == 31u) {
                    // Every 32 tiles: publish this list's kc-th and (kc / 4)-th scores (a list's
                    // entries only improve, so both only rise) and take up a better floor from
                    // the query's lists: the best kc-th, or the 4th highest of the (kc / 4)-th
                    // scores (four lists then hold kc / 4 entries each at or above it).
                    std::uint32_t key;
                    if (count == p.kc) {
                        const std::uint32_t mine = float_to_key(list_d[(p.kc - 1) * kBM + e]);
                        key = max(atomicMax(p.floor_key + row, mine), mine);
                    } else {
                        key = __ldcg(p.floor_key + row);
                    }
                    const std::uint32_t quarter = p.kc >> 2;
                    std::uint32_t* qk = p.quarter_key + static_cast<std::size_t>(row) * lists;
                    if (count >= quarter) {
                        __stcg(qk + ch * p.halves + half, float_to_key(list_d[(quarter - 1) * kBM + e]));
                    }
                    std::uint32_t k0 = 0, k1 = 0, k2 = 0, k3 = 0;  // the four highest, k0 >= .. >= k3
                    for (std::uint32_t l = 0; l < lists; ++l) {
                        std::uint32_t v = __ldcg(qk + l);
                        std::uint32_t m = max(k0, v);
                        v = min(k0, v);
                        k0 = m;
                        m = max(k1, v);
                        v = min(k1, v);
                        k1 = m;
                        m = max(k2, v);
                        v = min(k2, v);
                        k2 = m;
                        k3 = max(k3, v);
                    }
                    key = max(key, k3);
                    const float fl = key_to_float(key);
                    if (fl > floor) {
                        floor = fl;
                        if (fl > thr) {
                            thr = fl;
                            thr_i = kNoId;
                        }
                    }
                }
            }
            if (!ok) {
                break;
            }
            if (live) {
                // Back to distances: d = ||q||^2 - t (L2) or 1 - t; order is preserved.
                const float qn = p.qnorm[row];
                const std::size_t list = static_cast<std::size_t>(row) * lists + ch * p.halves + half;
                const std::size_t at = list * p.kc;
                for (std::uint32_t i = 0; i < p.kc; ++i) {
                    const float v = list_d[i * kBM + e];
                    p.cand_d[at + i] = i < count ? (l2 ? __fsub_rn(qn, v) : __fsub_rn(1.0F, v)) : INFINITY;
                    p.cand_ids[at + i] = i < count ? list_i[i * kBM + e] : kNoId;
                }
                // Every excluded row of this item scored at most `thr` (the floor, or the full
                // list's kc-th, whichever is higher; both only rose): no excluded distance is
                // below the matching distance.
                const float bound = count == p.kc ? fmaxf(thr, floor) : floor;
                p.cand_tau[list] =
                    bound == -INFINITY ? INFINITY : (l2 ? __fsub_rn(qn, bound) : __fsub_rn(1.0F, bound));
                if (count == p.kc) {
                    atomicMax(p.floor_key + row, float_to_key(list_d[(p.kc - 1) * kBM + e]));
                }
                if (count >= (p.kc >> 2)) {
                    __stcg(p.quarter_key + static_cast<std::size_t>(row) * lists + ch * p.halves + half,
                           float_to_key(list_d[((p.kc >> 2) - 1) * kBM + e]));
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols)
                     : "memory");
    }
}

// -------------------------------------------------------------------------------------------
// Preparation: bf16 hi / lo split, norms, flags. One warp per row.

__device__ __forceinline__ bool small_integer(float v) {
    return v == rintf(v) && fabsf(v) <= 256.0F;
}

struct PrepOut {
    __nv_bfloat16* hi;
    __nv_bfloat16* lo;
    float* norm;
    float* normalized;        // FP32 rows as searched (queries only; may be null)
    std::uint8_t* exact;      // per row: small-integer components (may be null)
    std::uint8_t* valid;      // per row (queries only)
    std::uint32_t* flags;     // bit 0: a nonzero lo part; bit 1: a row that is not small-integer
    float* max_norm;          // max sqrt(norm) (as u32 bits, atomicMax)
    std::uint32_t* status;    // queries: error code, first bad row
};

__global__ void prep_rows_kernel(const float* src, std::uint32_t src_stride, std::uint32_t rows,
                                 std::uint32_t dim, std::uint32_t dk, std::uint32_t row32,
                                 std::uint32_t metric, std::uint32_t check, PrepOut o) {
    const int lane = threadIdx.x & 31;
    const std::uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    extern __shared__ __align__(16) float qbuf[];
    float* q = qbuf + (threadIdx.x >> 5) * row32;
    for (std::uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += warps) {
        const float* x = src + static_cast<std::size_t>(r) * src_stride;
        bool bad = false;
        for (std::uint32_t e = lane; e < row32; e += 32) {
            const float v = e < dim ? x[e] : 0.0F;
            bad |= !isfinite(v);
            q[e] = v;
        }
        __syncwarp();
        bool valid = true;
        if (check && __any_sync(kFull, bad)) {
            if (lane == 0) {
                atomicCAS(o.status, 0u, 1u);
                atomicMin(o.status + 1, r);
            }
            valid = false;
        } else if (check && metric == 2) {
            const float raw = warp_raw<kFP32, false>(q, reinterpret_cast<const unsigned char*>(q),
                                                     dim, row32 * 4, lane);
            const float n = sqrtf(raw);
            if (!(n > 0.0F) || !isfinite(n)) {
                if (lane == 0) {
                    atomicCAS(o.status, 0u, 2u);
                    atomicMin(o.status + 1, r);
                }
                valid = false;
            } else {
                __syncwarp();
                for (std::uint32_t e = lane; e < dim; e += 32) {
                    q[e] = __fdiv_rn(q[e], n);
                }
            }
        }
        __syncwarp();
        bool has_lo = false, not_int = false;
        for (std::uint32_t e = lane; e < dk; e += 32) {
            const float v = valid && e < dim ? q[e] : 0.0F;
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
            has_lo |= __bfloat162float(l) != 0.0F;
            not_int |= !small_integer(v);
            o.hi[static_cast<std::size_t>(r) * dk + e] = h;
            o.lo[static_cast<std::size_t>(r) * dk + e] = l;
            if (o.normalized != nullptr && e < row32) {
                o.normalized[static_cast<std::size_t>(r) * row32 + e] = valid ? q[e] : 0.0F;
            }
        }
        has_lo = __any_sync(kFull, has_lo);
        not_int = __any_sync(kFull, not_int);
        __syncwarp();
        const float nrm = valid ? warp_raw<kFP32, false>(q, reinterpret_cast<const unsigned char*>(q),
                                                         dim, row32 * 4, lane)
                                : 0.0F;
        if (lane == 0) {
            o.norm[r] = nrm;
            if (o.exact != nullptr) {
                o.exact[r] = not_int ? 0 : 1;
            }
            if (o.valid != nullptr) {
                o.valid[r] = valid ? 1 : 0;
            }
            const std::uint32_t f = (has_lo ? 1u : 0u) | (not_int ? 2u : 0u);
            if (f != 0) {
                atomicOr(o.flags, f);
            }
            atomicMax(reinterpret_cast<std::uint32_t*>(o.max_norm), __float_as_uint(sqrtf(nrm)));
        }
        __syncwarp();
    }
}

// The epilogue's per-row score offset, added to c * q.x: -||x||^2 for L2, -0 for inner product
// (so the score is q.x - 0 exactly), -inf past the end.
__global__ void bias_kernel(const float* norm, float* bias, std::uint32_t n, std::uint32_t n_pad,
                            std::uint32_t l2) {
    const std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_pad) {
        bias[i] = i < n ? (l2 ? -norm[i] : -0.0F) : -INFINITY;
    }
}

// -------------------------------------------------------------------------------------------
// Merge, exact re-rank, certification. One warp per query.

struct MergeParams {
    std::uint32_t nq, n, dim, row32, lists, kc, k, out_stride, metric, dk, terms;
    const float* queries;          // normalized FP32 rows [nq][row32]
    const std::uint8_t* valid;
    const std::uint8_t* q_exact;
    const float* qnorm;
    const float* vectors;          // FP32 stored rows [n][row32]
    std::uint32_t base_exact;      // every stored component a small integer
    const float* xmax;             // max stored norm
    const std::uint32_t* cand_ids;
    const float* cand_d;
    const float* cand_tau;
    std::uint32_t* out_ids;
    float* out_dists;
    std::uint32_t* out_counts;
    std::uint32_t* uncertified;    // [nq] rows, count in uncertified_count
    std::uint32_t* uncertified_count;
    const std::uint32_t* status;   // the call's status word (nonzero: the call has failed)
};

template <bool kL2>
__global__ void bf_tc_merge_kernel(const MergeParams p) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const std::uint32_t per_warp = p.row32 * 4 + p.kc * 16 + 128;
    unsigned char* ws = sm + warp * per_warp;
    float* q = reinterpret_cast<float*>(ws);
    float* rd = reinterpret_cast<float*>(ws + p.row32 * 4);
    std::uint32_t* rid = reinterpret_cast<std::uint32_t*>(ws + p.row32 * 4 + p.kc * 4);
    float* ed = reinterpret_cast<float*>(ws + p.row32 * 4 + p.kc * 8);
    std::uint32_t* eid = reinterpret_cast<std::uint32_t*>(ws + p.row32 * 4 + p.kc * 12);
    int* ap = reinterpret_cast<int*>(ws + p.row32 * 4 + p.kc * 16);
    const std::uint32_t row = blockIdx.x * (blockDim.x >> 5) + warp;
    // After a failed scoring pass (a timed-out wait) the candidate lists were never written:
    // nothing here may read them (their stale contents are no valid merge input), and the call
    // reports the failure.
    if (row >= p.nq || *p.status != 0) {
        return;
    }
    std::uint32_t* oid = p.out_ids + static_cast<std::size_t>(row) * p.out_stride;
    float* od = p.out_dists + static_cast<std::size_t>(row) * p.out_stride;
    if (!p.valid[row]) {
        for (std::uint32_t i = lane; i < p.out_stride; i += 32) {
            oid[i] = kNoId;
            od[i] = INFINITY;
        }
        if (lane == 0) {
            p.out_counts[row] = 0;
        }
        return;
    }
    for (std::uint32_t e = lane; e < p.row32; e += 32) {
        q[e] = p.queries[static_cast<std::size_t>(row) * p.row32 + e];
    }
    __syncwarp();
    int r = 0;
    float tau = INFINITY;
    unsigned long long unused = 0;
    for (std::uint32_t ch = 0; ch < p.lists; ++ch) {
        const std::size_t at = (static_cast<std::size_t>(row) * p.lists + ch) * p.kc;
        for (std::uint32_t j0 = 0; j0 < p.kc; j0 += 32) {
            // kc may be 16: lanes past this list's end read nothing.
            const bool in = j0 + lane < p.kc;
            const std::uint32_t id = in ? p.cand_ids[at + j0 + lane] : kNoId;
            const float d = in ? p.cand_d[at + j0 + lane] : INFINITY;
            merge_round(rd, rid, r, static_cast<int>(p.kc), d, id, id < p.n, ap, lane, unused);
        }
        tau = fminf(tau, p.cand_tau[static_cast<std::size_t>(row) * p.lists + ch]);
    }
    if (r == static_cast<int>(p.kc)) {
        tau = fminf(tau, rd[r - 1]);  // every candidate dropped here was at least this far
    }
    // Exact distances of the kept candidates, in the reference's order.
    float my_d = INFINITY;
    std::uint32_t my_id = kNoId;
    int rr = 0;
    for (int j0 = 0; j0 < r; j0 += 32) {
        const int j = j0 + lane;
        const bool valid = j < r;
        if (valid) {
            my_id = rid[j] & kIdMask;
            my_d = lane_distance<kFP32, kL2>(
                q, reinterpret_cast<const unsigned char*>(p.vectors + static_cast<std::size_t>(my_id) * p.row32),
                p.dim, p.row32 * 4);
        }
        __syncwarp();
        merge_round(ed, eid, rr, static_cast<int>(p.k), my_d, my_id, valid, ap, lane, unused);
    }
    const int cnt = rr;
    // Certification: no excluded vector can have an exact distance at or below the k-th.
    bool certified = true;
    if (tau < INFINITY) {
        if (cnt < static_cast<int>(p.k)) {
            certified = false;
        } else {
            const float ek = ed[cnt - 1];
            float eps;
            if (p.base_exact && p.q_exact[row] && p.metric == 0) {
                eps = tau * 0x1.0p-23F;  // exact arithmetic; one rounding above 2^24
            } else {
                const float a = sqrtf(p.qnorm[row]) + *p.xmax;
                const float c = 0x1.0p-13F + static_cast<float>(p.terms * p.dk + 2 * p.dim + 8) * 0x1.0p-22F;
                eps = c * a * a;
            }
            certified = ek < tau - eps;
        }
    }
    for (std::uint32_t i = lane; i < p.out_stride; i += 32) {
        if (static_cast<int>(i) < cnt) {
            oid[i] = eid[i] & kIdMask;
            od[i] = ed[i];
        } else {
            oid[i] = kNoId;
            od[i] = INFINITY;
        }
    }
    if (lane == 0) {
        p.out_counts[row] = static_cast<std::uint32_t>(cnt);
        if (!certified) {
            const std::uint32_t at = atomicAdd(p.uncertified_count, 1u);
            p.uncertified[at] = row;
        }
    }
}

// -------------------------------------------------------------------------------------------
// Host side

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
    static EncodeTiled fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            return static_cast<EncodeTiled>(nullptr);
        }
        return reinterpret_cast<EncodeTiled>(f);
    }();
    return fn;
}

// A [rows][dk] bf16 row-major matrix as 64 x 128 boxes with 128-byte swizzling.
bool make_map(CUtensorMap* map, const void* ptr, std::uint32_t rows, std::uint32_t dk) {
    EncodeTiled enc = encoder();
    if (enc == nullptr) {
        return false;
    }
    const cuuint64_t dims[2] = {dk, rows};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(dk) * 2};
    const cuuint32_t box[2] = {kBK, kBM};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box,
               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

std::size_t align_up(std::size_t x, std::size_t a) { return (x + a - 1) / a * a; }

// The pipeline-wait limit of the next launches (nanoseconds; kWaitNs unless a test set it).
std::atomic<std::uint64_t> g_tc_wait_ns{kWaitNs};

struct Plan {
    std::uint32_t dk, kchunks, kc, stages, qtiles, nchunks, tpq, grid, halves;
    std::uint32_t off_b, off_lists, off_bar;
    std::size_t smem;
    bool ok;
};

Plan make_plan(std::uint32_t nq, std::uint32_t n, std::uint32_t dim, std::uint32_t k, bool xlo,
               int sms) {
    Plan pl{};
    pl.dk = static_cast<std::uint32_t>(align_up(dim, kBK));
    pl.kchunks = pl.dk / kBK;
    pl.kc = k <= 10 ? 16 : (k <= 24 ? 32 : (k <= 48 ? 64 : 0));
    pl.ok = pl.kc != 0 && pl.kchunks <= 4 && n >= 1;
    if (!pl.ok) {
        return pl;
    }
    const std::size_t a_bytes = 2 * pl.kchunks * kChunk;
    const std::size_t stage = (xlo ? 2 : 1) * pl.kchunks * kChunk;
    const std::size_t limit = 227 * 1024 - 1024 - 256;
    // Two epilogue halves (two candidate lists per row) when they fit beside at least two
    // pipeline stages; otherwise one.
    std::uint32_t stages = 0;
    std::size_t lists = 0;
    for (pl.halves = 2; pl.halves >= 1; --pl.halves) {
        lists = static_cast<std::size_t>(pl.halves) * pl.kc * kBM * 8;
        stages = 4;
        while (stages > 1 && a_bytes + stages * stage + lists > limit) {
            --stages;
        }
        if (a_bytes + stages * stage + lists <= limit && stages >= 2) {
            break;
        }
    }
    if (pl.halves == 0) {
        pl.ok = false;
        return pl;
    }
    pl.stages = stages;
    pl.off_b = static_cast<std::uint32_t>(a_bytes);
    pl.off_lists = static_cast<std::uint32_t>(a_bytes + stages * stage);
    pl.off_bar = static_cast<std::uint32_t>(pl.off_lists + lists);
    pl.smem = 1024 + pl.off_bar + 8 * (2 * stages) + 64 + 16;
    pl.qtiles = (nq + kBM - 1) / kBM;
    // Chunks of the stored rows: the fewest whose (query tile, chunk) items fill the waves of
    // one CTA per SM to 97 % (the last wave's idle SMs are the loss), else the best filling.
    pl.tpq = (n + kBN - 1) / kBN;
    const std::uint32_t most = std::min<std::uint32_t>(pl.tpq, 2u * static_cast<std::uint32_t>(sms));
    double best = 0.0;
    pl.nchunks = 1;
    for (std::uint32_t c = 1; c <= most; ++c) {
        const std::uint64_t items = static_cast<std::uint64_t>(pl.qtiles) * c;
        const std::uint64_t waves = (items + sms - 1) / sms;
        const double fill = static_cast<double>(items) / static_cast<double>(waves * sms);
        if (fill > best + 1e-9) {
            best = fill;
            pl.nchunks = c;
        }
        if (fill >= 0.97) {
            break;
        }
    }
    pl.grid = static_cast<std::uint32_t>(std::min<std::uint64_t>(
        static_cast<std::uint64_t>(pl.qtiles) * pl.nchunks, static_cast<std::uint64_t>(sms)));
    return pl;
}

}  // namespace

std::uint64_t tc_wait_ns() { return g_tc_wait_ns.load(); }
void set_tc_wait_ns(std::uint64_t ns) { g_tc_wait_ns.store(ns == 0 ? kWaitNs : ns); }

struct TcBase {
    void* hi = nullptr;
    void* lo = nullptr;
    float* norm = nullptr;
    void* flags = nullptr;   // [0] flags, [1] max norm bits
    float* bias = nullptr;   // [n rounded up to a tile]: ||x||^2 (L2) or 0 (IP); +inf padding
    std::uint32_t n = 0, dk = 0;
    bool has_lo = false, exact = false;
    float max_norm = 0.0F;
    CUtensorMap map_hi{}, map_lo{};
    int device = 0;
};

void free_tc_base(TcBase* b) {
    if (b == nullptr) {
        return;
    }
    for (void* ptr : {b->hi, b->lo, static_cast<void*>(b->norm), b->flags, static_cast<void*>(b->bias)}) {
        if (ptr != nullptr) {
            cudaFree(ptr);
        }
    }
    delete b;
}

cudaError_t prepare_tc_base(const BaseView& v, cudaStream_t stream, TcBase** out) {
    auto* b = new TcBase();
    b->n = v.n;
    b->dk = static_cast<std::uint32_t>(align_up(v.dim, kBK));
    cudaGetDevice(&b->device);
    const std::size_t elems = static_cast<std::size_t>(v.n) * b->dk;
    const std::size_t n_pad = align_up(v.n, kBN);
    cudaError_t err = cudaMalloc(&b->hi, elems * 2);
    if (err == cudaSuccess) err = cudaMalloc(&b->lo, elems * 2);
    if (err == cudaSuccess) err = cudaMalloc(&b->norm, n_pad * 4);
    if (err == cudaSuccess) err = cudaMalloc(&b->bias, n_pad * 4);
    if (err == cudaSuccess) err = cudaMalloc(&b->flags, 16);
    if (err == cudaSuccess) err = cudaMemsetAsync(b->flags, 0, 16, stream);
    if (err != cudaSuccess) {
        free_tc_base(b);
        return err;
    }
    PrepOut o{};
    o.hi = static_cast<__nv_bfloat16*>(b->hi);
    o.lo = static_cast<__nv_bfloat16*>(b->lo);
    o.norm = b->norm;
    o.flags = static_cast<std::uint32_t*>(b->flags);
    o.max_norm = reinterpret_cast<float*>(static_cast<std::uint32_t*>(b->flags) + 1);
    const int warps = 8;
    prep_rows_kernel<<<1184, warps * 32, warps * v.row32 * 4, stream>>>(
        v.vectors, v.row32, v.n, v.dim, b->dk, v.row32, v.metric, 0, o);
    err = cudaGetLastError();
    if (err == cudaSuccess) {
        bias_kernel<<<(static_cast<unsigned>(n_pad) + 255) / 256, 256, 0, stream>>>(
            b->norm, b->bias, v.n, static_cast<std::uint32_t>(n_pad), v.metric == 0 ? 1u : 0u);
        err = cudaGetLastError();
    }
    std::uint32_t host_flags[2] = {0, 0};
    if (err == cudaSuccess) err = cudaMemcpyAsync(host_flags, b->flags, 8, cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err != cudaSuccess) {
        free_tc_base(b);
        return err;
    }
    b->has_lo = (host_flags[0] & 1u) != 0;
    // Exact integer arithmetic needs 2 * dim * 256^2 <= 2^24.
    b->exact = (host_flags[0] & 2u) == 0 && 2ull * v.dim * 65536ull <= (1ull << 24);
    std::memcpy(&b->max_norm, &host_flags[1], 4);
    if (!make_map(&b->map_hi, b->hi, v.n, b->dk) || !make_map(&b->map_lo, b->lo, v.n, b->dk)) {
        free_tc_base(b);
        return cudaErrorNotSupported;
    }
    *out = b;
    return cudaSuccess;
}

std::size_t bruteforce_tc_workspace(std::uint32_t nq, std::uint32_t n, std::uint32_t dim,
                                    std::uint32_t k) {
    const std::uint32_t dk = static_cast<std::uint32_t>(align_up(dim, kBK));
    const std::uint32_t row32 = static_cast<std::uint32_t>(align_up(dim, 4));
    const std::size_t nqp = align_up(nq, kBM);
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const Plan pl = make_plan(nq, n, dim, k, true, sms);
    // Candidate lists per query: chunks x column halves. The launch's plan may use two halves
    // where this one (sized for the largest stage) uses one, and the chunk count depends only on
    // the shapes, so size for two.
    const std::size_t chunks = pl.ok ? static_cast<std::size_t>(pl.nchunks) * 2 : 1;
    const std::size_t kc = pl.ok ? pl.kc : 32;
    return 4 * nqp * dk                         // q hi + lo
           + 4 * nqp * row32                    // normalized FP32 queries
           + 4 * nqp * 3                        // norms, exact and valid flags
           + nq * chunks * kc * 8 + nq * chunks * 8  // candidates, bounds, quarter keys
           + 8 * nqp + 4096 + 16 * 256;         // uncertified rows, floors, flags, alignment
}

cudaError_t launch_bruteforce_tc(const BruteArgs& a, const TcBase& b, void* workspace,
                                 cudaStream_t stream, std::uint32_t* uncertified_out) {
    if (a.nq == 0) {
        return cudaSuccess;
    }
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const std::uint32_t dim = a.base.dim, row32 = a.base.row32, nq = a.nq, n = a.base.n;
    Plan pl = make_plan(nq, n, dim, a.k, b.has_lo, sms);
    if (!pl.ok || a.k > n || a.qstride != dim) {
        return launch_bruteforce_exact(a, stream);  // shapes this path does not cover
    }
    const std::size_t nqp = align_up(nq, kBM);
    auto* w = static_cast<unsigned char*>(workspace);
    std::size_t off = 0;
    const auto take = [&](std::size_t bytes) {
        unsigned char* p = w + off;
        off = align_up(off + bytes, 256);
        return p;
    };
    auto* q_hi = reinterpret_cast<__nv_bfloat16*>(take(nqp * pl.dk * 2));
    auto* q_lo = reinterpret_cast<__nv_bfloat16*>(take(nqp * pl.dk * 2));
    auto* qf = reinterpret_cast<float*>(take(nqp * row32 * 4));
    auto* qnorm = reinterpret_cast<float*>(take(nqp * 4));
    auto* q_exact = take(nqp);
    auto* q_valid = take(nqp);
    const std::size_t lists = static_cast<std::size_t>(pl.nchunks) * pl.halves;
    auto* cand_ids = reinterpret_cast<std::uint32_t*>(take(static_cast<std::size_t>(nq) * lists * pl.kc * 4));
    auto* cand_d = reinterpret_cast<float*>(take(static_cast<std::size_t>(nq) * lists * pl.kc * 4));
    auto* cand_tau = reinterpret_cast<float*>(take(static_cast<std::size_t>(nq) * lists * 4));
    auto* uncert = reinterpret_cast<std::uint32_t*>(take(nqp * 4));
    auto* floor_key = reinterpret_cast<std::uint32_t*>(take(nqp * 4));
    auto* quarter_key = reinterpret_cast<std::uint32_t*>(take(static_cast<std::size_t>(nq) * lists * 4));
    auto* flags = reinterpret_cast<std::uint32_t*>(take(64));  // [0] query flags [1] max norm [2] error

    cudaError_t err = cudaMemsetAsync(flags, 0, 64, stream);
    // Zero keys decode to -inf: no floor yet.
    if (err == cudaSuccess) err = cudaMemsetAsync(floor_key, 0, nqp * 4, stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(quarter_key, 0, static_cast<std::size_t>(nq) * lists * 4, stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(uncertified_out, 0, 4, stream);
    if (err == cudaSuccess && nqp > nq) {
        err = cudaMemsetAsync(q_hi + static_cast<std::size_t>(nq) * pl.dk, 0, (nqp - nq) * pl.dk * 2, stream);
    }
    if (err == cudaSuccess && nqp > nq) {
        err = cudaMemsetAsync(q_lo + static_cast<std::size_t>(nq) * pl.dk, 0, (nqp - nq) * pl.dk * 2, stream);
    }
    if (err != cudaSuccess) {
        return err;
    }
    PrepOut o{};
    o.hi = q_hi;
    o.lo = q_lo;
    o.norm = qnorm;
    o.normalized = qf;
    o.exact = q_exact;
    o.valid = q_valid;
    o.flags = flags;
    o.max_norm = reinterpret_cast<float*>(flags + 1);
    o.status = a.status;
    prep_rows_kernel<<<std::min<std::uint32_t>((nq + 7) / 8, 1184), 256, 8 * row32 * 4, stream>>>(
        a.queries, a.qstride, nq, dim, pl.dk, row32, a.base.metric, 1, o);
    if ((err = cudaGetLastError()) != cudaSuccess) {
        return err;
    }

    CUtensorMap mq_hi, mq_lo;
    if (!make_map(&mq_hi, q_hi, static_cast<std::uint32_t>(nqp), pl.dk) ||
        !make_map(&mq_lo, q_lo, static_cast<std::uint32_t>(nqp), pl.dk)) {
        return cudaErrorNotSupported;
    }
    TcParams p{};
    p.nq = nq;
    p.n = n;
    p.dim = dim;
    p.kchunks = pl.kchunks;
    p.qtiles = pl.qtiles;
    p.nchunks = pl.nchunks;
    p.halves = pl.halves;
    p.tpq = pl.tpq;
    p.kc = pl.kc;
    p.stages = pl.stages;
    p.metric = a.base.metric == 0 ? 0u : 1u;
    p.base_lo = b.has_lo ? 1u : 0u;
    p.query_flags = flags;
    p.qnorm = qnorm;
    p.xnorm = b.bias;
    p.cand_ids = cand_ids;
    p.cand_d = cand_d;
    p.cand_tau = cand_tau;
    p.floor_key = floor_key;
    p.quarter_key = quarter_key;
    p.error = a.status;
    p.wait_ns = tc_wait_ns();
    p.off_b = pl.off_b;
    p.off_lists = pl.off_lists;
    p.off_bar = pl.off_bar;
    {
        int device = 0;
        err = cudaGetDevice(&device);
        if (err == cudaSuccess) {
            err = raise_smem_limit(reinterpret_cast<const void*>(&bf_tc_kernel), device, pl.smem);
        }
    }
    if (err != cudaSuccess) {
        return err;
    }
    bf_tc_kernel<<<pl.grid, kThreads, pl.smem, stream>>>(mq_hi, mq_lo, b.map_hi, b.map_lo, p);
    if ((err = cudaGetLastError()) != cudaSuccess) {
        return err;
    }

    MergeParams m{};
    m.nq = nq;
    m.n = n;
    m.dim = dim;
    m.row32 = row32;
    m.lists = static_cast<std::uint32_t>(lists);  // candidate lists per query
    m.kc = pl.kc;
    m.k = a.k;
    m.out_stride = a.out_stride;
    m.metric = a.base.metric;
    m.dk = pl.dk;
    m.terms = 3;  // hi*hi + hi*lo + lo*hi: the bound covers every term the data may need
    m.queries = qf;
    m.valid = q_valid;
    m.q_exact = q_exact;
    m.qnorm = qnorm;
    m.vectors = a.base.vectors;
    m.base_exact = b.exact ? 1u : 0u;
    m.cand_ids = cand_ids;
    m.cand_d = cand_d;
    m.cand_tau = cand_tau;
    m.out_ids = a.out_ids;
    m.out_dists = a.out_dists;
    m.out_counts = a.out_counts;
    m.uncertified = uncert;
    m.uncertified_count = uncertified_out;
    m.status = a.status;
    // The stored vectors' largest norm, as the prep kernel left it in the base's flag words.
    m.xmax = reinterpret_cast<const float*>(static_cast<const std::uint32_t*>(b.flags) + 1);
    const int warps = 8;
    const std::size_t msmem = static_cast<std::size_t>(warps) * (row32 * 4 + pl.kc * 16 + 128);
    if (a.base.metric == 0) {
        bf_tc_merge_kernel<true><<<(nq + warps - 1) / warps, warps * 32, msmem, stream>>>(m);
    } else {
        bf_tc_merge_kernel<false><<<(nq + warps - 1) / warps, warps * 32, msmem, stream>>>(m);
    }
    if ((err = cudaGetLastError()) != cudaSuccess) {
        return err;
    }

    // Queries the tensor cores could not certify: the exact kernel on just those rows.
    BruteArgs f = a;
    f.rows = uncert;
    f.nrows_device = uncertified_out;
    if ((err = launch_bruteforce_exact(f, stream)) != cudaSuccess) {
        return err;
    }
    return cudaSuccess;
}

}  // namespace vdx::dev
