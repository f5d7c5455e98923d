#pragma once

// Device helpers shared by the search and brute-force kernels: 16-byte asynchronous copies into
// shared memory, element loads for the three traversal precisions, and the warp distance.
//
// The warp distance reproduces the reference's AVX2 summation order (src/kernels_avx2.cpp:17-80
// of the reference) bit for bit, so FP32 GPU distances equal the reference's exactly:
//   lane L (0..31) is accumulator lane (j = L / 8, l = L % 8) and runs one FMA chain over the
//   elements 32t + L of every full 32-element block; lanes 0..7 then continue over the
//   remaining full 8-element blocks. The reduction is a butterfly whose partners are the
//   reference's: xor 8 gives acc0 + acc1 (and acc2 + acc3), xor 16 gives
//   (acc0 + acc1) + (acc2 + acc3), then xor 4, 2, 1 are the fixed horizontal tree
//   ((v0 + v4) + (v2 + v6)) + ((v1 + v5) + (v3 + v7)). IEEE addition is commutative, so every
//   lane ends with the same bits. The dim % 8 tail is summed by every lane in order; when it
//   has four or more elements its first four products are rounded before being added (the
//   reference's GCC 13.3 -O3 build vectorizes them), the others are single FMAs.
// Every rounding here is explicit (__fmaf_rn, __fmul_rn, __fadd_rn, __fsub_rn), so no compiler
// contraction can change a result.

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cstdint>

namespace vdx::dev {

constexpr std::uint32_t kNoId = 0xFFFFFFFFu;
constexpr std::uint32_t kFull = 0xFFFFFFFFu;

enum : int { kFP32 = 0, kBF16 = 1, kFP8 = 2 };

// Raises `kernel`'s dynamic shared-memory limit on `device` to at least `smem` bytes and never
// lowers it: the limit belongs to the device's context and is shared by every host thread, so a
// launch that set it to its own smaller size could make another thread's larger launch fail.
// Every kernel launched with a varying dynamic shared-memory size sets it through here.
// Defined in search.cu.
cudaError_t raise_smem_limit(const void* kernel, int device, std::size_t smem);

__device__ __forceinline__ std::uint32_t smem_addr(const void* p) {
    return static_cast<std::uint32_t>(__cvta_generic_to_shared(p));
}

// One 16-byte global -> shared copy, bypassing L1 (cp.async.cg), or with kL1 through L1
// (cp.async.ca: for data many warps of an SM read, like the upper layers' rows). Both addresses
// 16-aligned.
template <bool kL1 = false>
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    if constexpr (kL1) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem_dst)),
                     "l"(gmem_src)
                     : "memory");
    } else {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem_dst)),
                     "l"(gmem_src)
                     : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
// Waits (in hardware, no spin loop) until at most N of this thread's groups are pending.
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Element e of a traversal row held in shared or global memory, as FP32. For FP8 rows the
// per-vector scale is the last float of the row and multiplies every element.
template <int P>
__device__ __forceinline__ float row_elem(const unsigned char* row, std::uint32_t e, float scale) {
    if constexpr (P == kFP32) {
        return reinterpret_cast<const float*>(row)[e];
    } else if constexpr (P == kBF16) {
        return __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(row)[e]);
    } else {
        const __nv_fp8_e4m3 v = reinterpret_cast<const __nv_fp8_e4m3*>(row)[e];
        return __fmul_rn(scale, static_cast<float>(v));
    }
}

template <int P>
__device__ __forceinline__ float row_scale(const unsigned char* row, std::uint32_t row_bytes) {
    if constexpr (P == kFP8) {
        return *reinterpret_cast<const float*>(row + row_bytes - 4);
    } else {
        return 1.0F;
    }
}

// The raw sum between the query (FP32, shared memory, `dim` floats) and one row, computed by
// the whole warp in the reference's order; every lane returns the same value. kL2: squared L2;
// otherwise <q, x>.
template <int P, bool kL2>
__device__ __forceinline__ float warp_raw(const float* q, const unsigned char* row,
                                          std::uint32_t dim, std::uint32_t row_bytes, int lane) {
    const float scale = row_scale<P>(row, row_bytes);
    const std::uint32_t blocks32 = dim >> 5;
    float acc = 0.0F;
#pragma unroll 4
    for (std::uint32_t t = 0; t < blocks32; ++t) {
        const std::uint32_t e = (t << 5) + static_cast<std::uint32_t>(lane);
        const float x = row_elem<P>(row, e, scale);
        const float y = q[e];
        if constexpr (kL2) {
            const float d = __fsub_rn(y, x);
            acc = __fmaf_rn(d, d, acc);
        } else {
            acc = __fmaf_rn(y, x, acc);
        }
    }
    std::uint32_t i = blocks32 << 5;
    const std::uint32_t blocks8 = (dim - i) >> 3;
    if (lane < 8) {
        for (std::uint32_t r = 0; r < blocks8; ++r) {
            const std::uint32_t e = i + (r << 3) + static_cast<std::uint32_t>(lane);
            const float x = row_elem<P>(row, e, scale);
            const float y = q[e];
            if constexpr (kL2) {
                const float d = __fsub_rn(y, x);
                acc = __fmaf_rn(d, d, acc);
            } else {
                acc = __fmaf_rn(y, x, acc);
            }
        }
    }
    i += blocks8 << 3;
    acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 8));
    acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 16));
    acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 4));
    acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 2));
    acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, 1));
    const std::uint32_t tail = dim - i;
    for (std::uint32_t j = 0; j < tail; ++j) {
        const float x = row_elem<P>(row, i + j, scale);
        const float y = q[i + j];
        const float a = kL2 ? __fsub_rn(y, x) : y;
        const float b = kL2 ? a : x;
        if (tail >= 4 && j < 4) {
            acc = __fadd_rn(acc, __fmul_rn(a, b));
        } else {
            acc = __fmaf_rn(a, b, acc);
        }
    }
    return acc;
}

// The ranking distance: squared L2, or 1 - <q, x> (inner product and cosine).
template <int P, bool kL2>
__device__ __forceinline__ float warp_distance(const float* q, const unsigned char* row,
                                               std::uint32_t dim, std::uint32_t row_bytes,
                                               int lane) {
    const float raw = warp_raw<P, kL2>(q, row, dim, row_bytes, lane);
    return kL2 ? raw : __fsub_rn(1.0F, raw);
}

// Sixteen bytes of a traversal row starting at element e, as FP32: 4 (FP32), 8 (BF16) or 16
// (FP8) elements. `row + e * sizeof(element)` must be 16-byte aligned.
template <int P>
struct Vec {
    static constexpr int kPerLoad = P == kFP32 ? 4 : (P == kBF16 ? 8 : 16);
};

template <int P>
__device__ __forceinline__ void load16(const unsigned char* row, std::uint32_t e, float scale,
                                       float* out) {
    if constexpr (P == kFP32) {
        const float4 v = *reinterpret_cast<const float4*>(row + 4 * e);
        out[0] = v.x;
        out[1] = v.y;
        out[2] = v.z;
        out[3] = v.w;
    } else if constexpr (P == kBF16) {
        const uint4 v = *reinterpret_cast<const uint4*>(row + 2 * e);
        const std::uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            out[2 * i] = __uint_as_float(w[i] << 16);
            out[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
        }
    } else {
        const uint4 v = *reinterpret_cast<const uint4*>(row + e);
        const std::uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const __half2_raw lo = __nv_cvt_fp8x2_to_halfraw2(
                static_cast<__nv_fp8x2_storage_t>(w[i] & 0xFFFFu), __NV_E4M3);
            const __half2_raw hi = __nv_cvt_fp8x2_to_halfraw2(
                static_cast<__nv_fp8x2_storage_t>(w[i] >> 16), __NV_E4M3);
            const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&lo));
            const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&hi));
            out[4 * i] = __fmul_rn(scale, a.x);
            out[4 * i + 1] = __fmul_rn(scale, a.y);
            out[4 * i + 2] = __fmul_rn(scale, b.x);
            out[4 * i + 3] = __fmul_rn(scale, b.y);
        }
    }
}

template <bool kL2>
__device__ __forceinline__ void accumulate(float& acc, float q, float x) {
    if constexpr (kL2) {
        const float d = __fsub_rn(q, x);
        acc = __fmaf_rn(d, d, acc);
    } else {
        acc = __fmaf_rn(q, x, acc);
    }
}

// The raw sum (squared L2, or <q, x>) between the query and one row, computed by ONE lane with
// the reference's 32 accumulator lanes held in its registers: the same chains, tree and tail as
// warp_raw, so the bits are the same, but no shuffles and no cross-lane dependency, so a warp
// scores up to 32 rows at once. q (FP32) and row are 16-byte aligned (shared or global memory).
template <int P, bool kL2>
__device__ __forceinline__ float lane_raw(const float* q, const unsigned char* row,
                                          std::uint32_t dim, std::uint32_t row_bytes) {
    constexpr int E = Vec<P>::kPerLoad;
    const float scale = row_scale<P>(row, row_bytes);
    float acc[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) {
        acc[l] = 0.0F;
    }
    std::uint32_t i = 0;
    for (; dim - i >= 32; i += 32) {
#pragma unroll
        for (int u = 0; u < 32; u += E) {
            float x[E];
            load16<P>(row, i + u, scale, x);
#pragma unroll
            for (int v = 0; v < E; v += 4) {
                const float4 qv = *reinterpret_cast<const float4*>(q + i + u + v);
                accumulate<kL2>(acc[u + v], qv.x, x[v]);
                accumulate<kL2>(acc[u + v + 1], qv.y, x[v + 1]);
                accumulate<kL2>(acc[u + v + 2], qv.z, x[v + 2]);
                accumulate<kL2>(acc[u + v + 3], qv.w, x[v + 3]);
            }
        }
    }
    for (; dim - i >= 8; i += 8) {
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            accumulate<kL2>(acc[v], q[i + v], row_elem<P>(row, i + v, scale));
        }
    }
    float h[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        h[l] = __fadd_rn(__fadd_rn(acc[l], acc[l + 8]), __fadd_rn(acc[l + 16], acc[l + 24]));
    }
    float s = __fadd_rn(__fadd_rn(__fadd_rn(h[0], h[4]), __fadd_rn(h[2], h[6])),
                        __fadd_rn(__fadd_rn(h[1], h[5]), __fadd_rn(h[3], h[7])));
    const std::uint32_t tail = dim - i;
    for (std::uint32_t j = 0; j < tail; ++j) {
        const float x = row_elem<P>(row, i + j, scale);
        const float y = q[i + j];
        const float a = kL2 ? __fsub_rn(y, x) : y;
        const float b = kL2 ? a : x;
        if (tail >= 4 && j < 4) {
            s = __fadd_rn(s, __fmul_rn(a, b));
        } else {
            s = __fmaf_rn(a, b, s);
        }
    }
    return s;
}

template <int P, bool kL2>
__device__ __forceinline__ float lane_distance(const float* q, const unsigned char* row,
                                               std::uint32_t dim, std::uint32_t row_bytes) {
    const float raw = lane_raw<P, kL2>(q, row, dim, row_bytes);
    return kL2 ? raw : __fsub_rn(1.0F, raw);
}

// Paired FP32 arithmetic (sm_100 f32x2): each half is rounded exactly like the scalar
// instruction, so a pair of accumulator chains gives the same bits as two scalar chains.
__device__ __forceinline__ std::uint64_t pack2(float a, float b) {
    std::uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void unpack2(std::uint64_t v, float& a, float& b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
// acc += (q - x)^2 (kL2) or acc += q * x, on two chains at once.
template <bool kL2>
__device__ __forceinline__ void accumulate2(std::uint64_t& acc, std::uint64_t q, std::uint64_t x) {
    if constexpr (kL2) {
        std::uint64_t d;
        asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(q), "l"(x));
        asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(acc) : "l"(d), "l"(acc));
    } else {
        asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(q), "l"(x));
    }
}

// acc += (x - q)^2 on two chains, x the two BF16 elements packed in w (element 2i in the low
// half): sm_100's mixed-precision subtract takes the BF16 operand as it is (its conversion to
// FP32 is exact) and rounds x - q once, like the FP32 subtract of the converted element, and
// (x - q)^2 has the bits of (q - x)^2. One instruction per element instead of a conversion plus
// half a paired subtract.
__device__ __forceinline__ void accumulate2_l2_bf16(std::uint64_t& acc, std::uint32_t w, float q0,
                                                    float q1) {
    std::uint64_t d;
    asm("{\n\t.reg .b16 lo, hi;\n\t.reg .f32 a, b;\n\tmov.b32 {lo, hi}, %1;\n\t"
        "sub.rn.f32.bf16 a, lo, %2;\n\tsub.rn.f32.bf16 b, hi, %3;\n\tmov.b64 %0, {a, b};\n\t}"
        : "=l"(d) : "r"(w), "f"(q0), "f"(q1));
    asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(acc) : "l"(d), "l"(acc));
}

// The raw sum between the query and one row, computed by TWO lanes: `half` 0 runs the
// reference's accumulator lanes 0..15 (elements 32t + 0..15), `half` 1 lanes 16..31 (elements
// 32t + 16..31), two chains per paired instruction. Half 0 also runs the 8-element blocks
// (accumulator lanes 0..7). The tree: each half forms acc[l] + acc[l + 8] for its lanes,
// half 1 hands its eight sums to half 0 (partner = lane + 16: call with the row's halves in
// lanes L and L + 16, every lane of the warp converged), which adds them as
// (acc[l] + acc[l+8]) + (acc[l+16] + acc[l+24]), runs the fixed horizontal tree and the tail in
// the reference's order. The result is valid in half 0's lane only. Same bits as lane_raw.
// kDim != 0: the dimension is known at compile time (equal to `dim`), so the loops unroll and the
// loads issue back to back (a lone warp's BF16 call at d = 128: ~570 instead of ~890 cycles).
template <int P, bool kL2, std::uint32_t kDim = 0>
__device__ __forceinline__ float pair_raw(const float* q, const unsigned char* row,
                                          std::uint32_t dim_arg, std::uint32_t row_bytes, int half) {
    const std::uint32_t dim = kDim != 0 ? kDim : dim_arg;
    constexpr int E = Vec<P>::kPerLoad;
    const float scale = row_scale<P>(row, row_bytes);
    std::uint64_t acc[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        acc[l] = 0;  // two +0.0f
    }
    const std::uint32_t off = 16u * static_cast<std::uint32_t>(half);
    const auto block32 = [&](std::uint32_t i) {
#pragma unroll
        for (int u = 0; u < 16; u += E) {
            if constexpr (P == kBF16 && kL2) {
                const uint4 w = *reinterpret_cast<const uint4*>(row + 2 * (i + off + u));
                const float4 qa = *reinterpret_cast<const float4*>(q + i + off + u);
                const float4 qb = *reinterpret_cast<const float4*>(q + i + off + u + 4);
                accumulate2_l2_bf16(acc[(u >> 1) + 0], w.x, qa.x, qa.y);
                accumulate2_l2_bf16(acc[(u >> 1) + 1], w.y, qa.z, qa.w);
                accumulate2_l2_bf16(acc[(u >> 1) + 2], w.z, qb.x, qb.y);
                accumulate2_l2_bf16(acc[(u >> 1) + 3], w.w, qb.z, qb.w);
                continue;
            }
            float x[E];
            load16<P>(row, i + off + u, scale, x);
#pragma unroll
            for (int v = 0; v < E && u + v < 16; v += 4) {
                const float4 qv = *reinterpret_cast<const float4*>(q + i + off + u + v);
                accumulate2<kL2>(acc[(u + v) >> 1], pack2(qv.x, qv.y), pack2(x[v], x[v + 1]));
                accumulate2<kL2>(acc[((u + v) >> 1) + 1], pack2(qv.z, qv.w), pack2(x[v + 2], x[v + 3]));
            }
        }
    };
    std::uint32_t i = 0;
    if constexpr (kDim != 0) {
#pragma unroll
        for (std::uint32_t b = 0; b < kDim / 32; ++b) {
            block32(32 * b);
        }
        i = kDim / 32 * 32;
    } else {
        for (; dim - i >= 32; i += 32) {
            block32(i);
        }
    }
    const std::uint32_t blocks8_end = i + ((dim - i) & ~7u);
    if (half == 0) {
        for (std::uint32_t j = i; j < blocks8_end; j += 8) {
#pragma unroll
            for (int v = 0; v < 8; v += 2) {
                accumulate2<kL2>(acc[v >> 1], pack2(q[j + v], q[j + v + 1]),
                                 pack2(row_elem<P>(row, j + v, scale), row_elem<P>(row, j + v + 1, scale)));
            }
        }
    }
    float a[16];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        unpack2(acc[l], a[2 * l], a[2 * l + 1]);
    }
    float h[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        h[l] = __fadd_rn(a[l], a[l + 8]);
    }
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        const float other = __shfl_down_sync(kFull, h[l], 16);
        h[l] = __fadd_rn(h[l], other);
    }
    float s = __fadd_rn(__fadd_rn(__fadd_rn(h[0], h[4]), __fadd_rn(h[2], h[6])),
                        __fadd_rn(__fadd_rn(h[1], h[5]), __fadd_rn(h[3], h[7])));
    const std::uint32_t tail = dim - blocks8_end;
    for (std::uint32_t j = 0; j < tail; ++j) {
        const float x = row_elem<P>(row, blocks8_end + j, scale);
        const float y = q[blocks8_end + j];
        const float av = kL2 ? __fsub_rn(y, x) : y;
        const float bv = kL2 ? av : x;
        if (tail >= 4 && j < 4) {
            s = __fadd_rn(s, __fmul_rn(av, bv));
        } else {
            s = __fmaf_rn(av, bv, s);
        }
    }
    return s;
}

template <int P, bool kL2, std::uint32_t kDim = 0>
__device__ __forceinline__ float pair_distance(const float* q, const unsigned char* row,
                                               std::uint32_t dim, std::uint32_t row_bytes,
                                               int half) {
    const float raw = pair_raw<P, kL2, kDim>(q, row, dim, row_bytes, half);
    return kL2 ? raw : __fsub_rn(1.0F, raw);
}

// The raw sum between the query and one row of dimension kDim (a multiple of 32), computed by
// FOUR lanes: quarter j runs the reference's accumulator lanes 8j..8j+7 (elements 32t + 8j..8j+7),
// two chains per paired instruction, so each lane does a quarter of the row (a round of at most
// 8 rows scores them in half the time of the two-lane form). The tree joins the quarters as
// the reference adds (acc[l] + acc[l+8]) + (acc[l+16] + acc[l+24]): quarter 1 hands its sums to
// quarter 0 and quarter 3 to quarter 2 (lane + 8), then quarter 2 to quarter 0 (lane + 16); the
// horizontal tree follows. Call with row r's quarters in lanes r, r + 8, r + 16, r + 24, every
// lane of the warp converged; the result is valid in quarter 0's lane. Same bits as pair_raw.
// FP32 and BF16 rows only (a 16-byte FP8 load would straddle two quarters).
template <int P, bool kL2, std::uint32_t kDim>
__device__ __forceinline__ float quad_raw(const float* q, const unsigned char* row, int quarter) {
    static_assert(kDim % 32 == 0 && kDim > 0, "quad_raw needs a dimension that is a multiple of 32");
    static_assert(P != kFP8, "quad_raw reads 8 elements per lane and block");
    std::uint64_t acc[4] = {0, 0, 0, 0};
    const std::uint32_t off = 8u * static_cast<std::uint32_t>(quarter);
#pragma unroll
    for (std::uint32_t b = 0; b < kDim / 32; ++b) {
        const std::uint32_t e = 32 * b + off;
        const float4 qa = *reinterpret_cast<const float4*>(q + e);
        const float4 qb = *reinterpret_cast<const float4*>(q + e + 4);
        if constexpr (P == kBF16 && kL2) {
            const uint4 w = *reinterpret_cast<const uint4*>(row + 2 * e);
            accumulate2_l2_bf16(acc[0], w.x, qa.x, qa.y);
            accumulate2_l2_bf16(acc[1], w.y, qa.z, qa.w);
            accumulate2_l2_bf16(acc[2], w.z, qb.x, qb.y);
            accumulate2_l2_bf16(acc[3], w.w, qb.z, qb.w);
        } else {
            float x[8];
            if constexpr (P == kBF16) {
                load16<P>(row, e, 1.0F, x);
            } else {
                load16<P>(row, e, 1.0F, x);
                load16<P>(row, e + 4, 1.0F, x + 4);
            }
            accumulate2<kL2>(acc[0], pack2(qa.x, qa.y), pack2(x[0], x[1]));
            accumulate2<kL2>(acc[1], pack2(qa.z, qa.w), pack2(x[2], x[3]));
            accumulate2<kL2>(acc[2], pack2(qb.x, qb.y), pack2(x[4], x[5]));
            accumulate2<kL2>(acc[3], pack2(qb.z, qb.w), pack2(x[6], x[7]));
        }
    }
    float a[8];
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        unpack2(acc[l], a[2 * l], a[2 * l + 1]);
    }
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        a[l] = __fadd_rn(a[l], __shfl_down_sync(kFull, a[l], 8));
    }
    float h[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        h[l] = __fadd_rn(a[l], __shfl_down_sync(kFull, a[l], 16));
    }
    return __fadd_rn(__fadd_rn(__fadd_rn(h[0], h[4]), __fadd_rn(h[2], h[6])),
                     __fadd_rn(__fadd_rn(h[1], h[5]), __fadd_rn(h[3], h[7])));
}

template <int P, bool kL2, std::uint32_t kDim>
__device__ __forceinline__ float quad_distance(const float* q, const unsigned char* row, int quarter) {
    const float raw = quad_raw<P, kL2, kDim>(q, row, quarter);
    return kL2 ? raw : __fsub_rn(1.0F, raw);
}

// A shared-memory row stride for `row_bytes` rows read one row per lane with 16-byte loads:
// an odd number of 16-byte units, so the 8 lanes of each load phase hit distinct banks.
__host__ __device__ __forceinline__ std::uint32_t padded_row_stride(std::uint32_t row_bytes) {
    return ((row_bytes >> 4) & 1u) ? row_bytes : row_bytes + 16;
}

// The same order computed by ONE thread over a whole row (32 accumulators in registers): the
// exact distance for brute-force re-ranking, where one thread owns one candidate.
template <bool kL2>
__device__ __forceinline__ float thread_distance(const float* q, const float* x,
                                                 std::uint32_t dim) {
    float acc[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) {
        acc[l] = 0.0F;
    }
    std::uint32_t i = 0;
    for (; dim - i >= 32; i += 32) {
#pragma unroll
        for (int l = 0; l < 32; ++l) {
            const float a = q[i + l];
            const float b = x[i + l];
            if constexpr (kL2) {
                const float d = __fsub_rn(a, b);
                acc[l] = __fmaf_rn(d, d, acc[l]);
            } else {
                acc[l] = __fmaf_rn(a, b, acc[l]);
            }
        }
    }
    for (; dim - i >= 8; i += 8) {
#pragma unroll
        for (int l = 0; l < 8; ++l) {
            const float a = q[i + l];
            const float b = x[i + l];
            if constexpr (kL2) {
                const float d = __fsub_rn(a, b);
                acc[l] = __fmaf_rn(d, d, acc[l]);
            } else {
                acc[l] = __fmaf_rn(a, b, acc[l]);
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

// (distance, id) order of the reference's `closer` (include/vecdex/neighbor.hpp:23-25).
__device__ __forceinline__ bool closer(float da, std::uint32_t ia, float db, std::uint32_t ib) {
    return da < db || (da == db && ia < ib);
}

// Order-preserving map of a float (never NaN) to u32: a < b exactly when key(a) < key(b).
__device__ __forceinline__ std::uint32_t order_key(float f) {
    const std::uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float order_key_value(std::uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}
// The warp's smallest (d, tie) pair in (distance, tie) order, in every lane: two redux.sync
// minima (the distance key, then the tie value among the lanes holding that distance).
__device__ __forceinline__ void warp_argmin(float d, std::uint32_t tie, float& best_d,
                                            std::uint32_t& best_tie) {
    const std::uint32_t kd = order_key(d);
    const std::uint32_t m = __reduce_min_sync(kFull, kd);
    best_tie = __reduce_min_sync(kFull, kd == m ? tie : 0xFFFFFFFFu);
    best_d = order_key_value(m);
}

// Entries of a sorted result list carry this bit once expanded (ids stay below 2^31).
constexpr std::uint32_t kExpanded = 0x80000000u;
constexpr std::uint32_t kIdMask = 0x7FFFFFFFu;

// Merges up to 32 scored candidates (lane j holds candidate j when `valid`) into the sorted list
// R[0, r) of capacity ef: R = top-ef(R + candidates), candidates equal to an entry of R dropped.
// Returns the lowest position a candidate was written to (or INT_MAX).
template <typename Count>
__device__ __forceinline__ int merge_round(float* rd, std::uint32_t* rid, int& r, int ef,
                                           float my_d, std::uint32_t my_id, bool valid,
                                           int* ap, int lane, Count& dups) {
    // A full list admits only candidates that beat its worst entry.
    if (valid && r >= ef) {
        valid = closer(my_d, my_id, rd[r - 1], rid[r - 1] & kIdMask);
    }
    int lo = 0;
    bool adm = false;
    if (valid) {
        int hi = r;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            // closer(R[mid], candidate); the id is read only on a distance tie.
            const float dm = rd[mid];
            const bool before = dm < my_d || (dm == my_d && (rid[mid] & kIdMask) < my_id);
            if (before) {
                lo = mid + 1;
            } else {
                hi = mid;
            }
        }
        adm = !(lo < r && (rid[lo] & kIdMask) == my_id);
    }
    const std::uint32_t dupmask = __ballot_sync(kFull, valid && !adm);
    if (lane == 0) {
        dups += __popc(dupmask);
    }
    const std::uint32_t am = __ballot_sync(kFull, adm);
    if (am == 0) {
        return 0x7FFFFFFF;
    }
    int rank = 0;
    for (std::uint32_t m = am; m != 0; m &= m - 1) {
        const int j = __ffs(m) - 1;
        const float dj = __shfl_sync(kFull, my_d, j);
        const std::uint32_t ij = __shfl_sync(kFull, my_id, j);
        rank += (adm && closer(dj, ij, my_d, my_id)) ? 1 : 0;
    }
    const int na = __popc(am);
    if (adm) {
        ap[rank] = lo;  // admitted positions in R, in closer order (non-decreasing)
    }
    __syncwarp();
    const int minpos = ap[0];
    // Shift R[minpos, r) right by the number of admitted candidates before each entry; chunks
    // move from the top down so no entry is overwritten before it is read.
    for (int c = (r - 1) >> 5; c >= 0 && (c << 5) + 31 >= minpos; --c) {
        const int i = (c << 5) + lane;
        int np = -1;
        float di = 0.0F;
        std::uint32_t ii = 0;
        if (i >= minpos && i < r) {
            di = rd[i];
            ii = rid[i];
            int a = 0, b = na;
            while (a < b) {
                const int m = (a + b) >> 1;
                if (ap[m] <= i) {
                    a = m + 1;
                } else {
                    b = m;
                }
            }
            np = i + a;
        }
        __syncwarp();
        if (np >= 0 && np < ef) {
            rd[np] = di;
            rid[np] = ii;
        }
        __syncwarp();
    }
    const int newpos = lo + rank;
    const bool keep = adm && newpos < ef;
    if (keep) {
        rd[newpos] = my_d;
        rid[newpos] = my_id;
    }
    r = min(ef, r + na);
    const int low = static_cast<int>(
        __reduce_min_sync(kFull, keep ? static_cast<std::uint32_t>(newpos) : 0x7FFFFFFFu));
    __syncwarp();
    return low;
}

}  // namespace vdx::dev
