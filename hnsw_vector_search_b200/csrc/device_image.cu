// The device mirror as a file: a sidecar next to a v1 index file whose sections are the FP32
// device arrays in their device layout, each 4096-byte aligned, so loading is a straight copy
// per section (no re-layout; a GPUDirect-Storage reader could DMA them as they are). The v1
// file (docs/FORMAT.md) stays the index of record: the sidecar names the graph it mirrors by an
// XXH64 of the graph and refuses any other.
//
// Layout (little-endian): a 4096-byte header
//   0  "VDXDEV01" (8 bytes)        8  version u32 (1)           12 metric u32
//   16 n u64                       24 dim u32   28 row32 u32    32 M u32    36 stride0 u32
//   40 stride_up u32               44 max_level u32             48 entry u32  52 reserved u32
//   56 upper blocks u64            64 graph hash u64 (XXH64 of vectors, levels, layer-0 and upper
//                                     blocks of the index, in that order)
//   72 4 x (offset u64, bytes u64): vectors32, links0, upper_at, links_up
// then the sections: n x row32 f32 (rows zero-padded to 16 bytes), n x stride0 u32 (links then
// 0xFFFFFFFF), n u32 (first upper block of each node), blocks x stride_up u32.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <format>
#include <fstream>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <vector>

#include "common.cuh"
#include "gpu_runtime.cuh"
#include "vdx/device.hpp"
#include "vdx/hnsw.hpp"
#include "../host/src/internal.hpp"

namespace vdx {
namespace {

constexpr char kMagic[8] = {'V', 'D', 'X', 'D', 'E', 'V', '0', '1'};
constexpr std::uint32_t kVersion = 1;
constexpr std::size_t kAlign = 4096;
constexpr std::size_t kHeader = 4096;

std::size_t align_up(std::size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

template <typename T>
void put(std::vector<unsigned char>& h, std::size_t at, T v) {
    std::memcpy(h.data() + at, &v, sizeof v);
}
template <typename T>
T get(const std::vector<unsigned char>& h, std::size_t at) {
    T v;
    std::memcpy(&v, h.data() + at, sizeof v);
    return v;
}

struct Layout {
    std::uint32_t row32, stride0, stride_up;
    std::uint64_t n, blocks;
    std::uint64_t off[4], bytes[4];
};

Layout layout_of(std::size_t n, std::size_t dim, std::size_t M, std::uint64_t blocks) {
    Layout l{};
    l.row32 = static_cast<std::uint32_t>((dim + 3) / 4 * 4);
    l.stride0 = static_cast<std::uint32_t>((2 * M + 3) / 4 * 4);
    l.stride_up = static_cast<std::uint32_t>((M + 3) / 4 * 4);
    l.n = n;
    l.blocks = blocks;
    l.bytes[0] = n * l.row32 * 4;
    l.bytes[1] = n * l.stride0 * 4;
    l.bytes[2] = n * 4;
    l.bytes[3] = blocks * l.stride_up * 4;
    std::size_t at = kHeader;
    for (int i = 0; i < 4; ++i) {
        l.off[i] = at;
        at = align_up(at + l.bytes[i]);
    }
    return l;
}

}  // namespace

std::uint64_t HnswIndex::graph_hash() const {
    detail::Xxh64 h;
    h.update(vectors_.data().data(), vectors_.data().size_bytes());
    h.update(levels_.data(), levels_.size());
    h.update(layer0_.data(), layer0_.size() * sizeof(Id));
    for (const auto& blocks : upper_) {
        h.update(blocks.data(), blocks.size() * sizeof(Id));
    }
    return h.digest();
}

void HnswIndex::save_device_image(const std::filesystem::path& path) const {
    const std::size_t n = size();
    const std::size_t M = params_.M;
    std::uint64_t blocks = 0;
    for (const auto level : levels_) {
        blocks += level;
    }
    const Layout l = layout_of(n, dim(), M, blocks);
    std::vector<unsigned char> header(kHeader, 0);
    std::memcpy(header.data(), kMagic, 8);
    put<std::uint32_t>(header, 8, kVersion);
    put<std::uint32_t>(header, 12, static_cast<std::uint32_t>(metric_));
    put<std::uint64_t>(header, 16, n);
    put<std::uint32_t>(header, 24, static_cast<std::uint32_t>(dim()));
    put<std::uint32_t>(header, 28, l.row32);
    put<std::uint32_t>(header, 32, static_cast<std::uint32_t>(M));
    put<std::uint32_t>(header, 36, l.stride0);
    put<std::uint32_t>(header, 40, l.stride_up);
    put<std::uint32_t>(header, 44, static_cast<std::uint32_t>(max_level_));
    put<std::uint32_t>(header, 48, entry_point_);
    put<std::uint64_t>(header, 56, blocks);
    put<std::uint64_t>(header, 64, graph_hash());
    for (int i = 0; i < 4; ++i) {
        put<std::uint64_t>(header, 72 + 16 * i, l.off[i]);
        put<std::uint64_t>(header, 80 + 16 * i, l.bytes[i]);
    }
    std::ofstream out(path, std::ios::binary | std::ios::trunc);
    if (!out) {
        throw std::runtime_error(std::format("{}: cannot open for writing", path.string()));
    }
    out.write(reinterpret_cast<const char*>(header.data()), static_cast<std::streamsize>(header.size()));
    const auto pad_to = [&](std::uint64_t at) {
        const std::uint64_t now = static_cast<std::uint64_t>(out.tellp());
        if (at > now) {
            std::vector<char> zeros(at - now, 0);
            out.write(zeros.data(), static_cast<std::streamsize>(zeros.size()));
        }
    };
    // Section 0: rows padded to row32.
    pad_to(l.off[0]);
    {
        std::vector<float> row(l.row32, 0.0F);
        for (std::size_t r = 0; r < n; ++r) {
            std::memcpy(row.data(), vector_of(static_cast<Id>(r)), dim() * 4);
            out.write(reinterpret_cast<const char*>(row.data()), l.row32 * 4);
        }
    }
    // Section 1: layer-0 blocks in the device layout.
    pad_to(l.off[1]);
    {
        std::vector<std::uint32_t> b(l.stride0);
        for (std::size_t v = 0; v < n; ++v) {
            const auto ids = links(static_cast<Id>(v), 0);
            std::fill(b.begin(), b.end(), dev::kNoId);
            std::copy(ids.begin(), ids.end(), b.begin());
            out.write(reinterpret_cast<const char*>(b.data()), l.stride0 * 4);
        }
    }
    // Sections 2 and 3: upper index and blocks.
    pad_to(l.off[2]);
    {
        std::uint32_t next = 0;
        for (std::size_t v = 0; v < n; ++v) {
            out.write(reinterpret_cast<const char*>(&next), 4);
            next += levels_[v];
        }
    }
    pad_to(l.off[3]);
    {
        std::vector<std::uint32_t> b(l.stride_up);
        for (std::size_t v = 0; v < n; ++v) {
            for (std::size_t layer = 1; layer <= levels_[v]; ++layer) {
                const auto ids = links(static_cast<Id>(v), layer);
                std::fill(b.begin(), b.end(), dev::kNoId);
                std::copy(ids.begin(), ids.end(), b.begin());
                out.write(reinterpret_cast<const char*>(b.data()), l.stride_up * 4);
            }
        }
    }
    if (!out) {
        throw std::runtime_error(std::format("{}: write failed", path.string()));
    }
}

void HnswIndex::load_device_image(const std::filesystem::path& path, int device) const {
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        throw std::runtime_error(std::format("{}: cannot open", path.string()));
    }
    std::vector<unsigned char> header(kHeader);
    in.read(reinterpret_cast<char*>(header.data()), kHeader);
    if (!in || std::memcmp(header.data(), kMagic, 8) != 0) {
        throw std::runtime_error(std::format("{}: not a vdx device image", path.string()));
    }
    if (get<std::uint32_t>(header, 8) != kVersion) {
        throw std::runtime_error(std::format("{}: device image version {} is not supported", path.string(),
                                             get<std::uint32_t>(header, 8)));
    }
    std::uint64_t blocks = 0;
    for (const auto level : levels_) {
        blocks += level;
    }
    const Layout l = layout_of(size(), dim(), params_.M, blocks);
    const bool same_shape = get<std::uint32_t>(header, 12) == static_cast<std::uint32_t>(metric_) &&
                            get<std::uint64_t>(header, 16) == size() &&
                            get<std::uint32_t>(header, 24) == dim() &&
                            get<std::uint32_t>(header, 32) == params_.M &&
                            get<std::uint32_t>(header, 44) == max_level_ &&
                            get<std::uint32_t>(header, 48) == entry_point_ &&
                            get<std::uint64_t>(header, 56) == blocks;
    bool same_layout = true;
    for (int i = 0; i < 4; ++i) {
        same_layout = same_layout && get<std::uint64_t>(header, 72 + 16 * i) == l.off[i] &&
                      get<std::uint64_t>(header, 80 + 16 * i) == l.bytes[i];
    }
    if (!same_shape || !same_layout || get<std::uint64_t>(header, 64) != graph_hash()) {
        throw std::runtime_error(std::format("{}: the device image belongs to another graph", path.string()));
    }
    if (size() >= (std::size_t{1} << 31)) {
        throw std::length_error("vdx: the GPU search holds at most 2^31 - 1 nodes");
    }
    if (params_.M > 64) {
        throw std::invalid_argument("vdx: the GPU search supports M up to 64");
    }

    gpu::use_device(device);
    auto dg = std::make_unique<DeviceGraph>();
    dg->device = device;
    void** dst[4] = {&dg->vectors32_alloc, &dg->links0_alloc, &dg->upper_at_alloc, &dg->links_up_alloc};
    const char* names[4] = {"vectors", "layer-0 links", "upper index", "upper links"};
    // Two pinned staging buffers: the file read into one overlaps the copy out of the other.
    constexpr std::size_t kChunk = std::size_t{32} << 20;
    cudaStream_t stream = gpu::workspace(device).stream;
    struct Staging {
        void* host[2] = {nullptr, nullptr};
        cudaEvent_t done[2] = {nullptr, nullptr};
        ~Staging() {
            for (int b = 0; b < 2; ++b) {
                if (done[b] != nullptr) {
                    cudaEventSynchronize(done[b]);
                    cudaEventDestroy(done[b]);
                }
                cudaFreeHost(host[b]);
            }
        }
    } staging;
    for (int b = 0; b < 2; ++b) {
        gpu::check(cudaMallocHost(&staging.host[b], kChunk), "cudaMallocHost");
        gpu::check(cudaEventCreateWithFlags(&staging.done[b], cudaEventDisableTiming), "cudaEventCreate");
    }
    int turn = 0;
    for (int i = 0; i < 4; ++i) {
        *dst[i] = gpu::device_alloc(std::max<std::uint64_t>(l.bytes[i], 4), names[i]);
        dg->bytes += l.bytes[i];
        in.seekg(static_cast<std::streamoff>(l.off[i]));
        for (std::uint64_t done = 0; done < l.bytes[i]; turn ^= 1) {
            const std::size_t part = static_cast<std::size_t>(std::min<std::uint64_t>(kChunk, l.bytes[i] - done));
            gpu::check(cudaEventSynchronize(staging.done[turn]), "device image staging");
            in.read(static_cast<char*>(staging.host[turn]), static_cast<std::streamsize>(part));
            if (!in) {
                throw std::runtime_error(std::format("{}: truncated device image", path.string()));
            }
            gpu::check(cudaMemcpyAsync(static_cast<unsigned char*>(*dst[i]) + done, staging.host[turn], part,
                                       cudaMemcpyHostToDevice, stream),
                       "upload device image");
            gpu::check(cudaEventRecord(staging.done[turn], stream), "device image staging");
            done += part;
        }
    }
    gpu::check(cudaStreamSynchronize(stream), "upload device image");
    DeviceGraphView& v = dg->view;
    v.n = static_cast<std::uint32_t>(size());
    v.dim = static_cast<std::uint32_t>(dim());
    v.row32 = l.row32;
    v.cap0 = static_cast<std::uint32_t>(2 * params_.M);
    v.stride0 = l.stride0;
    v.cap_up = static_cast<std::uint32_t>(params_.M);
    v.stride_up = l.stride_up;
    v.max_level = static_cast<std::uint32_t>(max_level_);
    v.entry = entry_point_;
    v.metric = static_cast<std::uint32_t>(metric_);
    v.precision = 0;
    v.vectors32 = static_cast<const float*>(dg->vectors32_alloc);
    v.vectors = v.vectors32;
    v.row_bytes = l.row32 * 4;
    v.links0 = static_cast<const std::uint32_t*>(dg->links0_alloc);
    v.upper_at = static_cast<const std::uint32_t*>(dg->upper_at_alloc);
    v.links_up = static_cast<const std::uint32_t*>(dg->links_up_alloc);
    gpu::attach_upper_copy(*this, *dg, stream);
    if (!device_mutex_) {
        device_mutex_ = std::make_unique<std::mutex>();
    }
    const std::scoped_lock lock(*device_mutex_);
    const std::size_t slot = static_cast<std::size_t>(device) * 3 + static_cast<std::size_t>(Precision::FP32);
    if (device_.size() <= slot) {
        device_.resize(slot + 1);
    }
    device_[slot] = std::move(dg);
}

}  // namespace vdx
