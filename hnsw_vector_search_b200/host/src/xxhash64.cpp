// XXH64, written from the xxHash specification (doc/xxhash_spec.md in the xxHash repository):
// four 64-bit lanes consume 32-byte stripes; the lanes converge, the length is added, the
// remaining bytes are folded in 8-, 4- and 1-byte steps, and an avalanche finishes. The index
// file's checksum (docs/FORMAT.md "Checksum") is XXH64 with seed 0 over every byte before it.

#include <bit>
#include <cstring>

#include "internal.hpp"

namespace vdx::detail {
namespace {

constexpr std::uint64_t P1 = 11400714785074694791ULL;
constexpr std::uint64_t P2 = 14029467366897019727ULL;
constexpr std::uint64_t P3 = 1609587929392839161ULL;
constexpr std::uint64_t P4 = 9650029242287828579ULL;
constexpr std::uint64_t P5 = 2870177450012600261ULL;

std::uint64_t load64(const unsigned char* p) noexcept {
    std::uint64_t v;
    std::memcpy(&v, p, 8);
    return v;  // the format is little-endian, like every host this builds for
}
std::uint32_t load32(const unsigned char* p) noexcept {
    std::uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}
std::uint64_t round(std::uint64_t acc, std::uint64_t input) noexcept {
    return std::rotl(acc + input * P2, 31) * P1;
}
std::uint64_t merge(std::uint64_t acc, std::uint64_t lane) noexcept {
    return (acc ^ round(0, lane)) * P1 + P4;
}

}  // namespace

Xxh64::Xxh64(std::uint64_t seed) noexcept
    : v_{seed + P1 + P2, seed + P2, seed, seed - P1}, buf_{}, seed_(seed) {}

void Xxh64::stripe(const unsigned char* p) noexcept {
    for (int i = 0; i < 4; ++i) {
        v_[i] = round(v_[i], load64(p + 8 * i));
    }
}

void Xxh64::update(const void* data, std::size_t size) noexcept {
    const auto* p = static_cast<const unsigned char*>(data);
    total_ += size;
    if (buffered_ > 0) {
        const std::size_t take = size < 32 - buffered_ ? size : 32 - buffered_;
        std::memcpy(buf_ + buffered_, p, take);
        buffered_ += take;
        p += take;
        size -= take;
        if (buffered_ < 32) {
            return;
        }
        stripe(buf_);
        buffered_ = 0;
    }
    while (size >= 32) {
        stripe(p);
        p += 32;
        size -= 32;
    }
    std::memcpy(buf_, p, size);
    buffered_ = size;
}

std::uint64_t Xxh64::digest() const noexcept {
    std::uint64_t h;
    if (total_ >= 32) {
        h = std::rotl(v_[0], 1) + std::rotl(v_[1], 7) + std::rotl(v_[2], 12) + std::rotl(v_[3], 18);
        for (int i = 0; i < 4; ++i) {
            h = merge(h, v_[i]);
        }
    } else {
        h = seed_ + P5;
    }
    h += total_;
    const unsigned char* p = buf_;
    std::size_t left = buffered_;
    for (; left >= 8; p += 8, left -= 8) {
        h = std::rotl(h ^ round(0, load64(p)), 27) * P1 + P4;
    }
    if (left >= 4) {
        h = std::rotl(h ^ (static_cast<std::uint64_t>(load32(p)) * P1), 23) * P2 + P3;
        p += 4;
        left -= 4;
    }
    for (; left > 0; ++p, --left) {
        h = std::rotl(h ^ (static_cast<std::uint64_t>(*p) * P5), 11) * P1;
    }
    h ^= h >> 33;
    h *= P2;
    h ^= h >> 29;
    h *= P3;
    h ^= h >> 32;
    return h;
}

std::uint64_t xxh64(const void* data, std::size_t size, std::uint64_t seed) noexcept {
    Xxh64 h(seed);
    h.update(data, size);
    return h.digest();
}

}  // namespace vdx::detail
