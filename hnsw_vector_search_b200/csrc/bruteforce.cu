// Exact brute-force k-nearest-neighbor search on CUDA cores: the reference's
// BruteForceIndex::search (src/brute_force.cpp:19-37, :68-84) for a whole batch at once.
//
// A block holds one query per warp and streams the stored vectors through shared memory in
// tiles of 32 rows (double-buffered 16-byte cp.async copies, so each tile is read from memory
// once per block, not once per query). Lane j scores tile row j against its warp's query with the
// reference's FP32 summation order (thread_distance4: the 32 accumulator lanes of the AVX2
// kernel held in one thread's registers), so every distance equals the reference's bit for bit,
// and merges the 32 scores into the warp's sorted top-k list under `closer`. The result is the
// reference's result exactly, ties included.
//
// This is the correctness anchor and the fallback of the tensor-core path (bruteforce_tc.cu),
// which recomputes here any query it cannot certify.

#include <cuda_runtime.h>

#include <cstdint>

#include "bruteforce.cuh"
#include "common.cuh"

namespace vdx::dev {
namespace {

constexpr int kTileRows = 32;

// The reference order for one (query, row) pair in one thread, reading both from shared memory
// with 16-byte loads. q and x are 16-byte aligned.
template <bool kL2>
__device__ __forceinline__ float thread_distance4(const float* q, const float* x,
                                                  std::uint32_t dim) {
    float acc[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) {
        acc[l] = 0.0F;
    }
    std::uint32_t i = 0;
    for (; dim - i >= 32; i += 32) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float4 xv = *reinterpret_cast<const float4*>(x + i + 4 * c);
            const float4 qv = *reinterpret_cast<const float4*>(q + i + 4 * c);
            const float xs[4] = {xv.x, xv.y, xv.z, xv.w};
            const float qs[4] = {qv.x, qv.y, qv.z, qv.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if constexpr (kL2) {
                    const float d = __fsub_rn(qs[u], xs[u]);
                    acc[4 * c + u] = __fmaf_rn(d, d, acc[4 * c + u]);
                } else {
                    acc[4 * c + u] = __fmaf_rn(qs[u], xs[u], acc[4 * c + u]);
                }
            }
        }
    }
    for (; dim - i >= 8; i += 8) {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const float4 xv = *reinterpret_cast<const float4*>(x + i + 4 * c);
            const float4 qv = *reinterpret_cast<const float4*>(q + i + 4 * c);
            const float xs[4] = {xv.x, xv.y, xv.z, xv.w};
            const float qs[4] = {qv.x, qv.y, qv.z, qv.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if constexpr (kL2) {
                    const float d = __fsub_rn(qs[u], xs[u]);
                    acc[4 * c + u] = __fmaf_rn(d, d, acc[4 * c + u]);
                } else {
                    acc[4 * c + u] = __fmaf_rn(qs[u], xs[u], acc[4 * c + u]);
                }
            }
        }
    }
    float v[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        v[l] = __fadd_rn(__fadd_rn(acc[l], acc[l + 8]), __fadd_rn(acc[l + 16], acc[l + 24]));
    }
    float s = __fadd_rn(__fadd_rn(__fadd_rn(v[0], v[4]), __fadd_rn(v[2], v[6])),
                        __fadd_rn(__fadd_rn(v[1], v[5]), __fadd_rn(v[3], v[7])));
    const std::uint32_t tail = dim - i;
    for (std::uint32_t j = 0; j < tail; ++j) {
        const float a0 = q[i + j];
        const float b0 = x[i + j];
        const float a = kL2 ? __fsub_rn(a0, b0) : a0;
        const float b = kL2 ? a : b0;
        if (tail >= 4 && j < 4) {
            s = __fadd_rn(s, __fmul_rn(a, b));
        } else {
            s = __fmaf_rn(a, b, s);
        }
    }
    return kL2 ? s : __fsub_rn(1.0F, s);
}

__device__ __forceinline__ void report(std::uint32_t* status, std::uint32_t code,
                                       std::uint32_t row) {
    atomicCAS(status, 0u, code);
    atomicMin(status + 1, row);
}

struct Layout {
    std::uint32_t row_s;    // floats per shared tile row (conflict-free for 16-byte loads)
    std::uint32_t q_bytes;  // per-warp query area
    std::uint32_t tile_bytes;
    std::uint32_t list_bytes;  // per-warp top-k list
    std::uint32_t kcap;
};

template <bool kL2>
__global__ void __launch_bounds__(1024) bf_exact_kernel(const BruteArgs a, const Layout L) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = static_cast<int>(threadIdx.x & 31);
    const int warp = static_cast<int>(threadIdx.x >> 5);
    const int warps = static_cast<int>(blockDim.x >> 5);
    const BaseView& B = a.base;

    float* tiles = reinterpret_cast<float*>(smem);  // [2][kTileRows][row_s]
    unsigned char* per_warp = smem + 2 * L.tile_bytes + warp * (L.q_bytes + L.list_bytes + 128);
    float* q = reinterpret_cast<float*>(per_warp);
    float* rd = reinterpret_cast<float*>(per_warp + L.q_bytes);
    std::uint32_t* rid = reinterpret_cast<std::uint32_t*>(per_warp + L.q_bytes + L.kcap * 4);
    int* ap = reinterpret_cast<int*>(per_warp + L.q_bytes + L.list_bytes);

    const std::uint32_t limit = a.nrows_device != nullptr ? *a.nrows_device : a.nq;
    const std::uint32_t slot = blockIdx.x * static_cast<std::uint32_t>(warps) + warp;
    const bool block_live = blockIdx.x * static_cast<std::uint32_t>(warps) < limit;
    if (!block_live) {
        return;  // whole block: no one waits at the barriers below
    }
    bool active = slot < limit;
    const std::uint32_t row = active ? (a.rows != nullptr ? a.rows[slot] : slot) : 0;

    // Query: load, check, normalize under cosine.
    if (active) {
        const float* src = a.queries + static_cast<std::size_t>(row) * a.qstride;
        bool bad = false;
        for (std::uint32_t e = lane; e < L.q_bytes / 4; e += 32) {
            const float v = e < B.dim ? src[e] : 0.0F;
            bad |= !isfinite(v);
            q[e] = v;
        }
        __syncwarp();
        if (__any_sync(kFull, bad)) {
            if (lane == 0) {
                report(a.status, 1u, row);
            }
            active = false;
        } else if (B.metric == 2) {
            const float raw = warp_raw<kFP32, false>(q, reinterpret_cast<const unsigned char*>(q),
                                                     B.dim, B.row32 * 4, lane);
            const float nrm = sqrtf(raw);
            if (!(nrm > 0.0F) || !isfinite(nrm)) {
                if (lane == 0) {
                    report(a.status, 2u, row);
                }
                active = false;
            } else {
                __syncwarp();
                for (std::uint32_t e = lane; e < B.dim; e += 32) {
                    q[e] = __fdiv_rn(q[e], nrm);
                }
            }
        }
        __syncwarp();
    }

    const int keep = static_cast<int>(a.k < B.n ? a.k : B.n);
    int r = 0;
    const std::uint32_t chunks_per_row = B.row32 / 4;
    const std::uint32_t tiles_total = (B.n + kTileRows - 1) / kTileRows;
    const auto load_tile = [&](std::uint32_t t, int buf) {
        float* dst = tiles + buf * (L.tile_bytes / 4);
        const std::uint32_t first = t * kTileRows;
        const std::uint32_t rows_here = B.n - first < kTileRows ? B.n - first : kTileRows;
        const std::uint32_t total = rows_here * chunks_per_row;
        for (std::uint32_t x = threadIdx.x; x < total; x += blockDim.x) {
            const std::uint32_t rr = x / chunks_per_row;
            const std::uint32_t c = x - rr * chunks_per_row;
            cp_async16(dst + rr * L.row_s + 4 * c,
                       B.vectors + static_cast<std::size_t>(first + rr) * B.row32 + 4 * c);
        }
        cp_async_commit();
    };
    unsigned long long unused = 0;
    if (tiles_total > 0) {
        load_tile(0, 0);
    }
    for (std::uint32_t t = 0; t < tiles_total; ++t) {
        cp_async_wait<0>();
        __syncthreads();
        if (t + 1 < tiles_total) {
            load_tile(t + 1, static_cast<int>((t + 1) & 1));
        }
        if (active) {
            const float* tile = tiles + (t & 1) * (L.tile_bytes / 4);
            const std::uint32_t id = t * kTileRows + lane;
            const bool valid = id < B.n;
            float d = INFINITY;
            if (valid) {
                d = thread_distance4<kL2>(q, tile + lane * L.row_s, B.dim);
            }
            merge_round(rd, rid, r, keep, d, id, valid, ap, lane, unused);
        }
        __syncthreads();  // the next iteration's load overwrites the buffer read here
    }
    cp_async_wait<0>();

    if (active) {
        std::uint32_t* oid = a.out_ids + static_cast<std::size_t>(row) * a.out_stride;
        float* od = a.out_dists + static_cast<std::size_t>(row) * a.out_stride;
        for (std::uint32_t i = lane; i < a.out_stride; i += 32) {
            if (static_cast<int>(i) < r) {
                oid[i] = rid[i] & kIdMask;
                od[i] = rd[i];
            } else {
                oid[i] = kNoId;
                od[i] = INFINITY;
            }
        }
        if (lane == 0) {
            a.out_counts[row] = static_cast<std::uint32_t>(r);
        }
    } else if (slot < limit && lane == 0) {
        a.out_counts[row] = 0;
    }
}

std::uint32_t round_up(std::uint32_t x, std::uint32_t m) { return (x + m - 1) / m * m; }

}  // namespace

cudaError_t launch_bruteforce_exact(const BruteArgs& a, cudaStream_t stream) {
    if (a.nq == 0) {
        return cudaSuccess;
    }
    Layout L{};
    L.row_s = a.base.row32 + ((4 + 32 - a.base.row32 % 32) % 32);
    L.tile_bytes = kTileRows * L.row_s * 4;
    L.q_bytes = round_up(a.base.row32, 4) * 4;
    std::uint32_t kcap = 32;
    const std::uint32_t keep = a.k < a.base.n ? a.k : a.base.n;
    while (kcap < keep) {
        kcap <<= 1;
    }
    L.kcap = kcap;
    L.list_bytes = kcap * 8;
    const std::uint32_t per_warp = L.q_bytes + L.list_bytes + 128;
    const std::uint32_t budget = 200 * 1024;
    int warps = 32;
    while (warps > 1 && 2 * L.tile_bytes + warps * per_warp > budget) {
        warps >>= 1;
    }
    const std::size_t smem = 2 * L.tile_bytes + static_cast<std::size_t>(warps) * per_warp;
    if (smem > budget) {
        return cudaErrorInvalidValue;  // k or dim too large for one block
    }
    const bool l2 = a.base.metric == 0;
    auto* kernel = l2 ? &bf_exact_kernel<true> : &bf_exact_kernel<false>;
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err == cudaSuccess) {
        err = raise_smem_limit(reinterpret_cast<const void*>(kernel), device, smem);
    }
    if (err != cudaSuccess) {
        return err;
    }
    const std::uint32_t blocks = (a.nq + warps - 1) / warps;
    kernel<<<blocks, warps * 32, smem, stream>>>(a, L);
    return cudaGetLastError();
}

}  // namespace vdx::dev
