#pragma once

// Metrics and the host-side distance functions.
//
// The host computes distances only while building a graph (HnswIndex::add) and normalizing
// stored vectors; every query distance is computed on the GPU. Both sides sum in the same fixed
// order, the reference's AVX2 kernel order (src/kernels_avx2.cpp:17-80 of the reference), so a
// graph built here is the graph the reference builds, and GPU distances equal the reference's
// bit for bit:
//   32-element blocks: 32 accumulator lanes, lane L running one FMA chain over elements 32t + L;
//   8-element blocks:  lanes 0..7 continue their chains;
//   reduction:         v_l = (a_l + a_{l+8}) + (a_{l+16} + a_{l+24}) for l < 8, then
//                      ((v0+v4) + (v2+v6)) + ((v1+v5) + (v3+v7));
//   tail (dim % 8):    sequential; when the tail has >= 4 elements its first four products are
//                      rounded before being added (the reference's GCC 13.3 -O3 build
//                      vectorizes them), every other tail term is one FMA.

#include <cstddef>
#include <cstdint>
#include <span>

namespace vdx {

// How an index compares vectors; smaller is closer. The file format's metric codes are these
// values (docs/FORMAT.md "Header" of the reference: 0 L2, 1 InnerProduct, 2 Cosine).
enum class Metric : std::uint8_t {
    L2 = 0,            // ||a - b||^2
    InnerProduct = 1,  // 1 - <a, b>
    Cosine = 2,        // 1 - <a, b> on unit vectors (indexes normalize stored vectors and queries)
};

float l2_squared(std::span<const float> a, std::span<const float> b) noexcept;
float inner_product(std::span<const float> a, std::span<const float> b) noexcept;
// The ranking distance under `metric`: l2_squared, or 1 - inner_product.
float distance(Metric metric, std::span<const float> a, std::span<const float> b) noexcept;

namespace detail {
float l2_squared_raw(const float* a, const float* b, std::size_t dim) noexcept;
float inner_product_raw(const float* a, const float* b, std::size_t dim) noexcept;
// "avx2" when the host kernels use AVX2+FMA instructions, "portable" otherwise. Both round
// identically.
const char* host_kernel_name() noexcept;
}  // namespace detail

}  // namespace vdx
