#pragma once

// Internal host helpers: argument validation with the reference's error messages
// (src/vector_ops.cpp:36-86 of the reference), normalization, and XXH64.

#include <cstddef>
#include <cstdint>
#include <span>
#include <string_view>
#include <vector>

#include "vdx/distance.hpp"

namespace vdx::detail {

struct IndexShape {
    Metric metric;
    std::size_t dim;
    std::size_t size;
};

bool all_finite(std::span<const float> values) noexcept;
bool can_normalize(std::span<const float> v) noexcept;
// v /= sqrt(<v, v>) elementwise with IEEE sqrt and division, <v, v> in the kernel order.
void normalize(std::span<float> v) noexcept;

// std::invalid_argument / std::length_error, messages prefixed with `where`.
void check_new_vectors(std::string_view where, const IndexShape& index, std::size_t given_dim,
                       std::span<const float> values);
// Host-side part of the query checks: dimension and k. Finiteness and (under cosine)
// normalizability are checked on the GPU as each query is loaded, and reported with the same
// messages (query_error_message).
void check_query_shape(std::string_view where, const IndexShape& index, std::size_t query_dim,
                       std::size_t k);
// The full check on the host, for the single-query search() entry.
void check_query(std::string_view where, const IndexShape& index, std::span<const float> query,
                 std::size_t k);

// XXH64 (xxHash 64-bit), written from the public specification (xxHash doc/xxhash_spec.md).
class Xxh64 {
public:
    explicit Xxh64(std::uint64_t seed = 0) noexcept;
    void update(const void* data, std::size_t size) noexcept;
    std::uint64_t digest() const noexcept;

private:
    void stripe(const unsigned char* p) noexcept;
    std::uint64_t v_[4];
    unsigned char buf_[32];
    std::size_t buffered_ = 0;
    std::uint64_t total_ = 0;
    std::uint64_t seed_;
};

std::uint64_t xxh64(const void* data, std::size_t size, std::uint64_t seed = 0) noexcept;

}  // namespace vdx::detail
