// Host distance kernels in the reference's AVX2 summation order (see vdx/distance.hpp).
// Compiled with -ffp-contract=off: every fused multiply-add here is explicit, so the compiler
// cannot change how anything rounds.

#include <cmath>
#include <cstddef>

#include "vdx/distance.hpp"

#if defined(__x86_64__) && defined(__GNUC__)
#include <immintrin.h>
#define VDX_HAVE_AVX2 1
#endif

namespace vdx::detail {
namespace {

// The tail of dim % 8 elements, starting at `i`, added onto `sum`.
template <bool kL2>
float tail(const float* a, const float* b, std::size_t i, std::size_t dim, float sum) noexcept {
    const std::size_t start = i;
    const bool split = dim - i >= 4;
    for (; i < dim; ++i) {
        const float x = kL2 ? a[i] - b[i] : a[i];
        const float y = kL2 ? x : b[i];
        if (split && i - start < 4) {
            const float p = x * y;
            sum = sum + p;
        } else {
            sum = std::fma(x, y, sum);
        }
    }
    return sum;
}

// Portable form: the same 32 chains and reduction tree, one lane at a time.
template <bool kL2>
float portable(const float* a, const float* b, std::size_t dim) noexcept {
    float acc[32] = {};
    std::size_t i = 0;
    for (; dim - i >= 32; i += 32) {
        for (std::size_t lane = 0; lane < 32; ++lane) {
            const float x = kL2 ? a[i + lane] - b[i + lane] : a[i + lane];
            const float y = kL2 ? x : b[i + lane];
            acc[lane] = std::fma(x, y, acc[lane]);
        }
    }
    for (; dim - i >= 8; i += 8) {
        for (std::size_t lane = 0; lane < 8; ++lane) {
            const float x = kL2 ? a[i + lane] - b[i + lane] : a[i + lane];
            const float y = kL2 ? x : b[i + lane];
            acc[lane] = std::fma(x, y, acc[lane]);
        }
    }
    float v[8];
    for (std::size_t l = 0; l < 8; ++l) {
        v[l] = (acc[l] + acc[l + 8]) + (acc[l + 16] + acc[l + 24]);
    }
    const float sum = ((v[0] + v[4]) + (v[2] + v[6])) + ((v[1] + v[5]) + (v[3] + v[7]));
    return tail<kL2>(a, b, i, dim, sum);
}

#ifdef VDX_HAVE_AVX2
template <bool kL2>
[[gnu::target("avx2,fma")]] float avx2(const float* a, const float* b, std::size_t dim) noexcept {
    __m256 acc[4] = {_mm256_setzero_ps(), _mm256_setzero_ps(), _mm256_setzero_ps(),
                     _mm256_setzero_ps()};
    std::size_t i = 0;
    for (; dim - i >= 32; i += 32) {
        for (int j = 0; j < 4; ++j) {
            const __m256 x = _mm256_loadu_ps(a + i + 8 * j);
            const __m256 y = _mm256_loadu_ps(b + i + 8 * j);
            if constexpr (kL2) {
                const __m256 d = _mm256_sub_ps(x, y);
                acc[j] = _mm256_fmadd_ps(d, d, acc[j]);
            } else {
                acc[j] = _mm256_fmadd_ps(x, y, acc[j]);
            }
        }
    }
    for (; dim - i >= 8; i += 8) {
        const __m256 x = _mm256_loadu_ps(a + i);
        const __m256 y = _mm256_loadu_ps(b + i);
        if constexpr (kL2) {
            const __m256 d = _mm256_sub_ps(x, y);
            acc[0] = _mm256_fmadd_ps(d, d, acc[0]);
        } else {
            acc[0] = _mm256_fmadd_ps(x, y, acc[0]);
        }
    }
    const __m256 v = _mm256_add_ps(_mm256_add_ps(acc[0], acc[1]), _mm256_add_ps(acc[2], acc[3]));
    alignas(32) float lanes[8];
    _mm256_store_ps(lanes, v);
    const float sum = ((lanes[0] + lanes[4]) + (lanes[2] + lanes[6])) +
                      ((lanes[1] + lanes[5]) + (lanes[3] + lanes[7]));
    return tail<kL2>(a, b, i, dim, sum);
}

bool cpu_has_avx2() noexcept {
    __builtin_cpu_init();
    return __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
}
#endif

using Fn = float (*)(const float*, const float*, std::size_t) noexcept;

struct Kernels {
    Fn l2;
    Fn ip;
    const char* name;
};

Kernels choose() noexcept {
#ifdef VDX_HAVE_AVX2
    if (cpu_has_avx2()) {
        return {&avx2<true>, &avx2<false>, "avx2"};
    }
#endif
    return {&portable<true>, &portable<false>, "portable"};
}

const Kernels& kernels() noexcept {
    static const Kernels k = choose();
    return k;
}

}  // namespace

float l2_squared_raw(const float* a, const float* b, std::size_t dim) noexcept {
    return kernels().l2(a, b, dim);
}
float inner_product_raw(const float* a, const float* b, std::size_t dim) noexcept {
    return kernels().ip(a, b, dim);
}
const char* host_kernel_name() noexcept { return kernels().name; }

}  // namespace vdx::detail

namespace vdx {

float l2_squared(std::span<const float> a, std::span<const float> b) noexcept {
    return detail::l2_squared_raw(a.data(), b.data(), a.size());
}
float inner_product(std::span<const float> a, std::span<const float> b) noexcept {
    return detail::inner_product_raw(a.data(), b.data(), a.size());
}
float distance(Metric metric, std::span<const float> a, std::span<const float> b) noexcept {
    return metric == Metric::L2 ? l2_squared(a, b) : 1.0F - inner_product(a, b);
}

}  // namespace vdx
