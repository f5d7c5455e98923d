#pragma once

// Launch interface of the exact brute-force kernels (bruteforce.cu, bruteforce_tc.cu).

#include <cuda_runtime.h>

#include <cstdint>

namespace vdx::dev {

// The stored vectors as the brute-force kernels read them: n rows of `row32` floats (dim rounded
// up to 4, zero padded; normalized under cosine, as the reference stores them).
struct BaseView {
    const float* vectors;
    std::uint32_t n;
    std::uint32_t dim;
    std::uint32_t row32;
    std::uint32_t metric;  // 0 L2, 1 inner product, 2 cosine
};

struct BruteArgs {
    BaseView base{};
    const float* queries = nullptr;   // nq rows of qstride floats
    std::uint32_t nq = 0;
    std::uint32_t qstride = 0;
    std::uint32_t k = 10;
    std::uint32_t out_stride = 10;
    std::uint32_t* out_ids = nullptr;
    float* out_dists = nullptr;
    std::uint32_t* out_counts = nullptr;
    std::uint32_t* status = nullptr;  // 2 words: error code, lowest failing row
    // Optional subset: only these query rows are searched (the fallback for rows the
    // tensor-core path could not certify).
    const std::uint32_t* rows = nullptr;
    const std::uint32_t* nrows_device = nullptr;
};

// Exact top-k by scanning every stored vector, every distance in the reference's FP32 order
// (bit-identical distances), the (distance, id) order of `closer`. CUDA cores.
cudaError_t launch_bruteforce_exact(const BruteArgs& args, cudaStream_t stream);

// Exact top-k through the tensor cores: a tcgen05 split-BF16 GEMM scores every pair, a fused
// epilogue keeps each query's best candidates per chunk, a merge keeps the best candidates
// overall, their distances are recomputed exactly (reference order), and a query is certified
// only if no excluded vector can beat its k-th exact distance under the scoring error bound;
// uncertified queries are recomputed by launch_bruteforce_exact. Shapes the path does not cover
// (k > 48, dim > 256, k > n) go to launch_bruteforce_exact directly.
//
// TcBase: the stored vectors prepared once (bf16 hi / lo, norms, flags, TMA descriptors).
struct TcBase;
cudaError_t prepare_tc_base(const BaseView& base, cudaStream_t stream, TcBase** out);
void free_tc_base(TcBase* base);
// `workspace` must hold bruteforce_tc_workspace() bytes; *uncertified_out (device) receives the
// number of queries recomputed exactly. A device wait that times out sets status code 5.
std::size_t bruteforce_tc_workspace(std::uint32_t nq, std::uint32_t n, std::uint32_t dim,
                                    std::uint32_t k);
cudaError_t launch_bruteforce_tc(const BruteArgs& args, const TcBase& base, void* workspace,
                                 cudaStream_t stream, std::uint32_t* uncertified_out);
// The limit of each pipeline wait of the next tensor-core launches, in nanoseconds (0 restores
// the default, 1 s). For tests of the timeout path; the drains before a CTA exits keep 1 s.
std::uint64_t tc_wait_ns();
void set_tc_wait_ns(std::uint64_t ns);

}  // namespace vdx::dev
