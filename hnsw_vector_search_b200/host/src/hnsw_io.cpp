// HnswIndex::save / load: the vecdex v1 index file (docs/FORMAT.md of the reference), so that
// files move between the reference and this library in both directions unchanged.
//
// The layout, the validation steps and their order, and the error messages follow the format
// specification and the reference's loader (src/hnsw_io.cpp:129-504), because a file the
// reference rejects must be rejected here with the same diagnosis. The reader is this project's
// own: the whole file is read into one buffer with one read, the checksum runs over it, and the
// sections are then copied out of it; the header is validated against the file size before
// anything proportional to a header field is allocated.

#include <fcntl.h>
#include <unistd.h>

#include <array>
#include <bit>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <format>
#include <limits>
#include <random>
#include <stdexcept>
#include <system_error>

#include "internal.hpp"
#include "vdx/hnsw.hpp"

namespace vdx {
namespace {

namespace fs = std::filesystem;

static_assert(std::endian::native == std::endian::little, "the index format is little-endian");

constexpr unsigned char kMagic[8] = {0x89, 'V', 'D', 'X', 'H', 'N', 'S', 'W'};
constexpr std::uint32_t kVersion = 1;
constexpr std::uint64_t kHeaderBytes = 80;
constexpr std::uint64_t kChecksumBytes = 8;

[[noreturn]] void fail(const fs::path& path, const std::string& what) {
    throw std::runtime_error(std::format("{}: {}", path.string(), what));
}

std::uint64_t mul(std::uint64_t a, std::uint64_t b, const fs::path& path) {
    if (b != 0 && a > std::numeric_limits<std::uint64_t>::max() / b) {
        fail(path, "the header's sizes overflow 64 bits");
    }
    return a * b;
}

std::uint64_t add(std::uint64_t a, std::uint64_t b, const fs::path& path) {
    if (a > std::numeric_limits<std::uint64_t>::max() - b) {
        fail(path, "the header's sizes overflow 64 bits");
    }
    return a + b;
}

template <typename T>
T field(const unsigned char* p) {
    T v;
    std::memcpy(&v, p, sizeof v);
    return v;
}

template <typename T>
void put(std::vector<unsigned char>& out, T v) {
    const auto* p = reinterpret_cast<const unsigned char*>(&v);
    out.insert(out.end(), p, p + sizeof v);
}

struct Header {
    std::uint32_t version, metric;
    std::uint64_t dim, M, ef_construction, seed, nodes, max_level, entry_point, upper_blocks;
};

Header parse_header(const unsigned char* h) {
    return {field<std::uint32_t>(h + 8),  field<std::uint32_t>(h + 12), field<std::uint64_t>(h + 16),
            field<std::uint64_t>(h + 24), field<std::uint64_t>(h + 32), field<std::uint64_t>(h + 40),
            field<std::uint64_t>(h + 48), field<std::uint64_t>(h + 56), field<std::uint64_t>(h + 64),
            field<std::uint64_t>(h + 72)};
}

// Checks each field, then that the sizes it implies sum exactly to the file size.
void check_header(const unsigned char* raw, const Header& h, std::uint64_t file_size,
                  const fs::path& path) {
    if (std::memcmp(raw, kMagic, 8) != 0) {
        fail(path, "not a vecdex HNSW index (wrong magic bytes)");
    }
    if (h.version != kVersion) {
        fail(path, std::format("format version {} is not supported (this build reads version {})",
                               h.version, kVersion));
    }
    if (h.metric > 2) {
        fail(path, std::format("unknown metric code {}", h.metric));
    }
    if (h.dim == 0) {
        fail(path, "dimension is 0");
    }
    if (h.M < 2) {
        fail(path, std::format("M is {}, below the minimum of 2", h.M));
    }
    if (h.M > HnswParams::kMaxM) {
        fail(path, std::format("M is {}, above the maximum of {}", h.M, HnswParams::kMaxM));
    }
    if (h.ef_construction == 0) {
        fail(path, "ef_construction is 0");
    }
    if (h.nodes > std::numeric_limits<Id>::max()) {
        fail(path, std::format("{} nodes is more than 32-bit ids can address", h.nodes));
    }
    if (h.max_level > 255) {
        fail(path, std::format("max level {} is above 255", h.max_level));
    }
    if (h.nodes == 0 && (h.max_level != 0 || h.entry_point != 0 || h.upper_blocks != 0)) {
        fail(path, "an empty index must have max level, entry point and upper blocks 0");
    }
    if (h.nodes > 0 && h.entry_point >= h.nodes) {
        fail(path, std::format("entry point {} is not one of the {} nodes", h.entry_point, h.nodes));
    }
    std::uint64_t expected = kHeaderBytes + kChecksumBytes;
    expected = add(expected, h.nodes, path);
    expected = add(expected, mul(mul(h.nodes, 1 + 2 * h.M, path), 4, path), path);
    expected = add(expected, mul(mul(h.upper_blocks, 1 + h.M, path), 4, path), path);
    expected = add(expected, mul(mul(h.nodes, h.dim, path), 4, path), path);
    if (expected != file_size) {
        fail(path, std::format("the header describes {} bytes but the file has {}; it is "
                               "truncated or corrupted",
                               expected, file_size));
    }
}

// Reads the whole file. Its size is known (and checked) before this is called.
std::vector<unsigned char> read_all(const fs::path& path, std::uint64_t size) {
    std::vector<unsigned char> bytes(size);
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (f == nullptr) {
        fail(path, "cannot open file");
    }
    const std::size_t got = std::fread(bytes.data(), 1, size, f);
    std::fclose(f);
    if (got != size) {
        fail(path, "unexpected end of file");
    }
    return bytes;
}

std::error_code flush(const fs::path& path, bool directory) {
    const int fd = ::open(path.c_str(), directory ? (O_RDONLY | O_DIRECTORY) : O_RDONLY);
    if (fd < 0) {
        return {errno, std::generic_category()};
    }
    int rc;
    do {
        rc = ::fsync(fd);
    } while (rc != 0 && errno == EINTR);
    const std::error_code ec = rc == 0 ? std::error_code{} : std::error_code{errno, std::generic_category()};
    ::close(fd);
    return ec;
}

}  // namespace

void HnswIndex::save(const std::filesystem::path& path) const {
    const bool empty = size() == 0;
    std::uint64_t upper = 0;
    for (const std::uint8_t l : levels_) {
        upper += l;
    }
    std::vector<unsigned char> out;
    out.reserve(kHeaderBytes + levels_.size() + (layer0_.size() + upper * (1 + params_.M)) * 4 +
                vectors_.data().size_bytes() + kChecksumBytes);
    out.insert(out.end(), kMagic, kMagic + 8);
    put<std::uint32_t>(out, kVersion);
    put<std::uint32_t>(out, static_cast<std::uint32_t>(metric_));
    for (const std::uint64_t v :
         {static_cast<std::uint64_t>(dim()), static_cast<std::uint64_t>(params_.M),
          static_cast<std::uint64_t>(params_.ef_construction), params_.seed,
          static_cast<std::uint64_t>(size()),
          empty ? std::uint64_t{0} : static_cast<std::uint64_t>(max_level_),
          empty ? std::uint64_t{0} : static_cast<std::uint64_t>(entry_point_), upper}) {
        put<std::uint64_t>(out, v);
    }
    out.insert(out.end(), levels_.begin(), levels_.end());
    const auto append_ids = [&out](std::span<const Id> ids) {
        const auto* p = reinterpret_cast<const unsigned char*>(ids.data());
        out.insert(out.end(), p, p + ids.size_bytes());
    };
    append_ids(layer0_);
    for (const auto& blocks : upper_) {
        append_ids(blocks);
    }
    const auto* vp = reinterpret_cast<const unsigned char*>(vectors_.data().data());
    out.insert(out.end(), vp, vp + vectors_.data().size_bytes());
    put<std::uint64_t>(out, detail::xxh64(out.data(), out.size()));

    // Atomic and durable replacement: write a fresh temporary next to `path`, flush it, rename
    // it over `path`, flush the directory.
    std::random_device rd;
    const std::uint64_t suffix = (std::uint64_t{rd()} << 32U) | rd();
    fs::path temp = path;
    temp += std::format(".tmp-{:016x}", suffix);
    std::FILE* f = std::fopen(temp.c_str(), "wb");
    if (f == nullptr) {
        fail(path, std::format("cannot create the temporary file {}", temp.string()));
    }
    const bool written = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    const bool closed = std::fclose(f) == 0;
    std::error_code ec;
    if (!written || !closed) {
        fs::remove(temp, ec);
        fail(path, std::format("cannot write the temporary file {}", temp.string()));
    }
    ec = flush(temp, false);
    if (ec) {
        std::error_code ignored;
        fs::remove(temp, ignored);
        fail(path, std::format("cannot flush the temporary file {} to storage: {}", temp.string(),
                               ec.message()));
    }
    fs::rename(temp, path, ec);
    if (ec) {
        std::error_code ignored;
        fs::remove(temp, ignored);
        fail(path, std::format("cannot replace it with {}: {}", temp.string(), ec.message()));
    }
    const fs::path dir = path.parent_path().empty() ? fs::path(".") : path.parent_path();
    ec = flush(dir, true);
    if (ec) {
        fail(path, std::format("saved, but cannot flush the directory {} to storage: {}",
                               dir.string(), ec.message()));
    }
}

HnswIndex HnswIndex::load(const std::filesystem::path& path) {
    std::error_code ec;
    const std::uintmax_t file_size = fs::file_size(path, ec);
    if (ec) {
        fail(path, ec.message());
    }
    if (file_size < kHeaderBytes + kChecksumBytes) {
        fail(path, std::format("{} bytes is too small for a vecdex index", file_size));
    }
    // The header alone first: nothing sized by its fields is allocated before they are checked
    // against the file size.
    unsigned char raw[kHeaderBytes];
    {
        std::FILE* f = std::fopen(path.c_str(), "rb");
        if (f == nullptr) {
            fail(path, "cannot open file");
        }
        const std::size_t got = std::fread(raw, 1, kHeaderBytes, f);
        std::fclose(f);
        if (got != kHeaderBytes) {
            fail(path, "unexpected end of file");
        }
    }
    const Header h = parse_header(raw);
    check_header(raw, h, file_size, path);

    const std::vector<unsigned char> bytes = read_all(path, file_size);
    if (detail::xxh64(bytes.data(), file_size - kChecksumBytes) !=
        field<std::uint64_t>(bytes.data() + file_size - kChecksumBytes)) {
        fail(path, "checksum mismatch: the file is corrupted");
    }
    const std::size_t n = h.nodes;
    const std::size_t b0 = 1 + 2 * h.M;
    const std::size_t b1 = 1 + h.M;
    const unsigned char* p = bytes.data() + kHeaderBytes;
    std::vector<std::uint8_t> levels(p, p + n);
    p += n;

    // Levels: each within the max level, summing to the header's block count, the entry point
    // on the top layer.
    std::uint64_t blocks = 0;
    for (std::size_t i = 0; i < n; ++i) {
        if (levels[i] > h.max_level) {
            fail(path, std::format("node {} has level {}, above the max level {}", i, levels[i],
                                   h.max_level));
        }
        blocks += levels[i];
    }
    if (blocks != h.upper_blocks) {
        fail(path, std::format("the levels add up to {} upper-layer blocks, but the header says {}",
                               blocks, h.upper_blocks));
    }
    if (n > 0 && levels[h.entry_point] != h.max_level) {
        fail(path, std::format("entry point {} has level {}, not the max level {}", h.entry_point,
                               levels[h.entry_point], h.max_level));
    }
    const unsigned char* layer0_at = p;
    const unsigned char* upper_at = layer0_at + n * b0 * 4;
    const unsigned char* vectors_at = upper_at + h.upper_blocks * b1 * 4;
    Matrix<float> vectors(n, h.dim);
    std::memcpy(vectors.data().data(), vectors_at, n * h.dim * 4);
    if (!detail::all_finite(vectors.data())) {
        fail(path, "a stored vector contains NaN or infinity");
    }

    HnswIndex index(h.dim, static_cast<Metric>(h.metric),
                    {.M = h.M, .ef_construction = h.ef_construction, .seed = h.seed});
    index.vectors_ = std::move(vectors);
    index.layer0_.resize(n * b0);
    std::memcpy(index.layer0_.data(), layer0_at, n * b0 * 4);
    index.upper_.reserve(n);
    const auto* up = reinterpret_cast<const Id*>(upper_at);  // memcpy'd below, never dereferenced
    std::size_t at = 0;
    for (std::size_t i = 0; i < n; ++i) {
        std::vector<Id> own(levels[i] * b1);
        std::memcpy(own.data(), upper_at + at * 4, own.size() * 4);
        at += own.size();
        index.upper_.push_back(std::move(own));
    }
    (void)up;
    index.levels_ = std::move(levels);
    index.entry_point_ = static_cast<Id>(h.entry_point);
    index.max_level_ = h.max_level;
    index.check_links(path);
    index.rng_.discard(n);  // each stored node drew its level once
    return index;
}

// Every block, before any link is followed: count within capacity; every id in range, not the
// node itself, living on that layer, and not repeated within the block.
void HnswIndex::check_links(const std::filesystem::path& path) const {
    const std::size_t n = size();
    std::vector<std::uint32_t> seen(n, 0);
    std::uint32_t stamp = 0;
    for (Id node = 0; node < n; ++node) {
        const std::size_t level = levels_[node];
        for (std::size_t layer = 0; layer <= level; ++layer) {
            const std::size_t count = block(node, layer)[0];
            if (count > max_links(layer)) {
                fail(path, std::format("node {} has {} links on layer {} (max {})", node, count,
                                       layer, max_links(layer)));
            }
            if (++stamp == 0) {
                std::ranges::fill(seen, 0U);
                stamp = 1;
            }
            for (const Id id : links(node, layer)) {
                if (id >= n) {
                    fail(path, std::format("node {} links to node {}, but there are only {} nodes",
                                           node, id, n));
                }
                if (id == node) {
                    fail(path, std::format("node {} links to itself on layer {}", node, layer));
                }
                if (levels_[id] < layer) {
                    fail(path, std::format("node {} links to node {} on layer {}, above its level {}",
                                           node, id, layer, levels_[id]));
                }
                if (seen[id] == stamp) {
                    fail(path,
                         std::format("node {} links to node {} twice on layer {}", node, id, layer));
                }
                seen[id] = stamp;
            }
        }
    }
}

}  // namespace vdx
