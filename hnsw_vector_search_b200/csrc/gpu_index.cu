// The host API's GPU side: device mirrors of an index, and the search entry points of
// HnswIndex and BruteForceIndex that run the kernels.
//
// Device mirrors are built on first use (and rebuilt after add()), under the index's mutex, so
// concurrent searches share one mirror. Each host thread keeps its own stream and its own
// device buffers for queries and results (thread_local, grown on demand), so concurrent
// searches never share scratch state, like the reference's scratch pool
// (src/search_scratch.hpp:61-105). Errors come back as the reference's exception types:
// std::invalid_argument for bad queries (with its messages), std::runtime_error for CUDA
// failures. There is no CPU search path: without a usable GPU every search throws.

#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <format>
#include <limits>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../host/src/internal.hpp"
#include "bruteforce.cuh"
#include "common.cuh"
#include "gpu_runtime.cuh"
#include "mlp.cuh"
#include "search.cuh"
#include "vdx/brute_force.hpp"
#include "vdx/device.hpp"
#include "vdx/hnsw.hpp"

namespace vdx {

struct DeviceBase {
    dev::BaseView view{};
    int device = 0;
    void* alloc = nullptr;
    mutable dev::TcBase* tc = nullptr;  // the tensor-core path's preparation, made on first use
    ~DeviceBase() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        dev::free_tc_base(tc);
        if (alloc != nullptr) {
            cudaFree(alloc);
        }
        cudaSetDevice(prev);
    }
};

DeviceGraph::~DeviceGraph() {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    for (void* p : {vectors_alloc, vectors32_alloc, links0_alloc, upper_at_alloc, links_up_alloc,
                    upper_copy_alloc}) {
        if (p != nullptr) {
            cudaFree(p);
        }
    }
    cudaSetDevice(prev);
}

namespace gpu {

void check(cudaError_t err, const char* what) {
    if (err != cudaSuccess) {
        throw CudaError(std::format("vdx: {}: CUDA error {} ({})", what, static_cast<int>(err),
                                    cudaGetErrorString(err)));
    }
}

void use_device(int device) {
    int count = 0;
    const cudaError_t err = cudaGetDeviceCount(&count);
    if (err != cudaSuccess || count == 0) {
        throw CudaError("vdx: no CUDA device is available; this library searches on the GPU only");
    }
    if (device < 0 || device >= count) {
        throw std::invalid_argument(std::format("vdx: device {} does not exist ({} found)", device, count));
    }
    check(cudaSetDevice(device), "cudaSetDevice");
}

namespace {

cudaMemPool_t order_pool(int device) {
    static std::mutex m;
    static std::vector<cudaMemPool_t> pools;
    const std::scoped_lock lock(m);
    if (pools.size() <= static_cast<std::size_t>(device)) {
        pools.resize(device + 1, nullptr);
    }
    if (pools[device] == nullptr) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        check(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
        std::uint64_t keep = ~std::uint64_t{0};
        check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
        pools[device] = pool;
    }
    return pools[device];
}

}  // namespace

OrderScratch::OrderScratch(int device, std::size_t nq, cudaStream_t stream) : nq_(nq), stream_(stream) {
    void* p = nullptr;
    check(cudaMallocFromPoolAsync(&p, std::max<std::size_t>(nq, 1) * 12, order_pool(device), stream),
          "order scratch");
    words_ = static_cast<std::uint32_t*>(p);
}

OrderScratch::~OrderScratch() {
    if (words_ != nullptr) {
        cudaFreeAsync(words_, stream_);
    }
}

const void* mapped_host(const void* host) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, host) != cudaSuccess) {
        cudaGetLastError();  // an unknown pointer is an answer here, not an error
        return nullptr;
    }
    return attr.type == cudaMemoryTypeHost ? attr.devicePointer : nullptr;
}

void* device_alloc(std::size_t bytes, const char* what) {
    void* p = nullptr;
    check(cudaMalloc(&p, bytes == 0 ? 16 : bytes), what);
    return p;
}

Workspace& workspace(int device) {
    thread_local std::vector<std::unique_ptr<Workspace>> per_device;
    if (per_device.size() <= static_cast<std::size_t>(device)) {
        per_device.resize(device + 1);
    }
    auto& ws = per_device[device];
    if (!ws) {
        ws = std::make_unique<Workspace>();
        ws->device = device;
        check(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ws->small = static_cast<std::uint32_t*>(device_alloc(256, "workspace"));
        check(cudaMallocHost(reinterpret_cast<void**>(&ws->small_host), 256), "cudaMallocHost");
    }
    return *ws;
}

Workspace::~Workspace() {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    for (void* p : {static_cast<void*>(queries), static_cast<void*>(ids), static_cast<void*>(dists),
                    static_cast<void*>(counts), static_cast<void*>(small), scratch, visited}) {
        if (p != nullptr) {
            cudaFree(p);
        }
    }
    if (small_host != nullptr) {
        cudaFreeHost(small_host);
    }
    if (stream != nullptr) {
        cudaStreamDestroy(stream);
    }
    cudaSetDevice(prev);
}

void Workspace::reserve(std::size_t nq, std::size_t dim, std::size_t width) {
    const auto grow = [](auto*& p, std::size_t& cap, std::size_t need, const char* what) {
        if (need > cap) {
            if (p != nullptr) {
                cudaFree(p);
                p = nullptr;
            }
            const std::size_t bytes = std::max<std::size_t>(need, 1) * sizeof(*p);
            p = static_cast<std::remove_reference_t<decltype(p)>>(device_alloc(bytes, what));
            cap = need;
        }
    };
    grow(queries, queries_cap, nq * dim, "query buffer");
    grow(ids, ids_cap, nq * width, "result ids");
    grow(dists, dists_cap, nq * width, "result distances");
    grow(counts, counts_cap, nq, "result counts");
}

void* Workspace::scratch_bytes(std::size_t bytes) {
    if (bytes > scratch_cap) {
        if (scratch != nullptr) {
            cudaFree(scratch);
        }
        scratch = device_alloc(bytes, "scratch");
        scratch_cap = bytes;
    }
    return scratch;
}

void* Workspace::visited_for(std::uint32_t slots, std::uint32_t warps) {
    if (visited == nullptr || slots > visited_stride || warps > visited_warps) {
        const std::uint32_t stride = std::max(slots, visited_stride);
        const std::uint32_t count = std::max(warps, visited_warps);
        const std::size_t bytes = dev::global_visited_bytes(stride, count);
        if (visited != nullptr) {
            check(cudaStreamSynchronize(stream), "visited tables");
            cudaFree(visited);
            visited = nullptr;
        }
        visited = device_alloc(bytes, "visited tables");
        check(cudaMemsetAsync(visited, 0, bytes, stream), "clear visited tables");
        visited_stride = stride;
        visited_warps = count;
    }
    return visited;
}

// Resets the status words (code 0, first bad row UINT32_MAX), the claim counter and the stats.
void reset_small(Workspace& ws) {
    check(cudaMemsetAsync(ws.small, 0, 256, ws.stream), "cudaMemsetAsync");
    check(cudaMemsetAsync(ws.small + 1, 0xFF, 4, ws.stream), "cudaMemsetAsync");
}

// Throws the reference's exception for a status word set by a kernel.
void raise_status(std::uint32_t code, const char* where) {
    switch (code) {
        case dev::kErrNone:
            return;
        case dev::kErrNonFinite:
            throw std::invalid_argument(std::format("{}: query must not contain NaN or inf", where));
        case dev::kErrZeroCosine:
            throw std::invalid_argument(
                std::format("{}: the cosine metric can't normalize a zero query", where));
        case dev::kErrBounds:
            throw DeviceBounds(std::format("{}: the device graph holds an out-of-range link", where));
        case dev::kErrCapacity:
            throw std::invalid_argument(std::format("{}: ef exceeds the GPU search capacity", where));
        case dev::kErrTimeout:
            throw DeviceTimeout(std::format("{}: a device wait timed out", where));
        default:
            throw std::runtime_error(std::format("{}: device error {}", where, code));
    }
}

namespace {

// Upper blocks with each id's upper_at beside it: block b of `stride` u32 becomes 2 * stride u32.
__global__ void upper_aug_kernel(const std::uint32_t* links_up, const std::uint32_t* upper_at,
                                 std::uint32_t* aug, std::uint32_t blocks, std::uint32_t stride,
                                 std::uint32_t n) {
    const std::size_t total = static_cast<std::size_t>(blocks) * stride;
    for (std::size_t x = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; x < total;
         x += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
        const std::size_t b = x / stride;
        const std::size_t j = x - b * stride;
        const std::uint32_t id = links_up[x];
        aug[b * 2 * stride + j] = id;
        // An id out of range (a corrupted mirror) keeps its slot, which the search reports; its
        // index is never read.
        const std::uint32_t ua = id < n ? upper_at[id] : 0u;
        aug[b * 2 * stride + stride + j] = ua < blocks ? ua : 0u;
    }
}

// The traversal row of every node with upper layers, at the index of its first upper block;
// 16 bytes per thread.
__global__ void upper_rows_kernel(const unsigned char* vectors, std::uint32_t row_bytes,
                                  const std::uint32_t* nodes, std::uint32_t count,
                                  const std::uint32_t* upper_at, unsigned char* rows,
                                  std::uint32_t blocks) {
    const std::uint32_t chunks = row_bytes >> 4;
    const std::size_t total = static_cast<std::size_t>(count) * chunks;
    for (std::size_t x = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; x < total;
         x += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
        const std::size_t i = x / chunks;
        const std::size_t c = x - i * chunks;
        const std::uint32_t node = nodes[i];
        const std::uint32_t ua = upper_at[node];
        if (ua < blocks) {
            const uint4 v = reinterpret_cast<const uint4*>(vectors + static_cast<std::size_t>(node) * row_bytes)[c];
            reinterpret_cast<uint4*>(rows + static_cast<std::size_t>(ua) * row_bytes)[c] = v;
        }
    }
}

}  // namespace

void attach_upper_copy(const HnswIndex& index, DeviceGraph& dg, cudaStream_t stream) {
    DeviceGraphView& v = dg.view;
    if (dg.upper_copy_alloc != nullptr) {
        cudaFree(dg.upper_copy_alloc);
        dg.upper_copy_alloc = nullptr;
    }
    v.upper_aug = nullptr;
    v.upper_rows = nullptr;
    v.l2_window = nullptr;
    v.l2_window_bytes = 0;
    const auto levels = index.levels();
    std::vector<std::uint32_t> nodes;
    std::uint32_t blocks = 0;
    std::uint32_t entry_ua = 0;
    for (std::uint32_t i = 0; i < levels.size(); ++i) {
        if (i == index.entry_point()) {
            entry_ua = blocks;
        }
        if (levels[i] > 0) {
            nodes.push_back(i);
        }
        blocks += levels[i];
    }
    if (blocks == 0 || v.max_level == 0) {
        return;
    }
    const std::size_t aug_bytes = (static_cast<std::size_t>(blocks) * 2 * v.stride_up * 4 + 255) / 256 * 256;
    const std::size_t rows_bytes = static_cast<std::size_t>(blocks) * v.row_bytes;
    dg.upper_copy_alloc = device_alloc(aug_bytes + rows_bytes, "upper-layer copy");
    dg.bytes += aug_bytes + rows_bytes;
    auto* base = static_cast<unsigned char*>(dg.upper_copy_alloc);
    void* d_nodes = device_alloc(nodes.size() * 4, "upper-layer nodes");
    check(cudaMemcpyAsync(d_nodes, nodes.data(), nodes.size() * 4, cudaMemcpyHostToDevice, stream),
          "upload upper-layer nodes");
    upper_aug_kernel<<<592, 256, 0, stream>>>(v.links_up, v.upper_at, reinterpret_cast<std::uint32_t*>(base),
                                             blocks, v.stride_up, v.n);
    check(cudaGetLastError(), "upper-layer copy");
    upper_rows_kernel<<<592, 256, 0, stream>>>(static_cast<const unsigned char*>(v.vectors), v.row_bytes,
                                              static_cast<const std::uint32_t*>(d_nodes),
                                              static_cast<std::uint32_t>(nodes.size()), v.upper_at,
                                              base + aug_bytes, blocks);
    check(cudaGetLastError(), "upper-layer copy");
    check(cudaStreamSynchronize(stream), "upper-layer copy");
    cudaFree(d_nodes);
    v.upper_aug = reinterpret_cast<const std::uint32_t*>(base);
    v.upper_rows = base + aug_bytes;
    v.entry_ua = entry_ua;
    // The L2 set-aside for persisting accesses (a limit of this process's context) is raised,
    // once per device, to cover the window where the device allows it.
    int max_persist = 0, max_window = 0;
    if (cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dg.device) == cudaSuccess &&
        cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dg.device) == cudaSuccess &&
        max_persist > 0 && max_window > 0) {
        static std::mutex limit_mutex;
        static std::size_t limit_set[64] = {};
        const std::scoped_lock lock(limit_mutex);
        const std::size_t window = std::min<std::size_t>(static_cast<std::size_t>(max_window),
                                                         aug_bytes + rows_bytes);
        const std::size_t want = std::min<std::size_t>(static_cast<std::size_t>(max_persist), window);
        if (dg.device >= 0 && dg.device < 64) {
            if (limit_set[dg.device] < want) {
                if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) == cudaSuccess) {
                    limit_set[dg.device] = want;
                } else {
                    cudaGetLastError();  // no set-aside: the window then only marks the rest streaming
                }
            }
            v.l2_window = base;
            v.l2_window_bytes = window;
            v.l2_hit_ratio = std::min(1.0F, static_cast<float>(limit_set[dg.device]) /
                                                static_cast<float>(window));
        }
    }
}

}  // namespace gpu

namespace {

std::uint32_t round_up(std::uint32_t x, std::uint32_t m) { return (x + m - 1) / m * m; }

// Layer-0 blocks [count, ids...] of stride 1 + cap -> fixed blocks of `stride`, unused slots
// 0xFFFFFFFF.
__global__ void repack_links_kernel(const std::uint32_t* src, std::uint32_t* dst, std::uint32_t n,
                                    std::uint32_t cap, std::uint32_t stride) {
    const std::size_t total = static_cast<std::size_t>(n) * stride;
    for (std::size_t x = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; x < total;
         x += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
        const std::size_t node = x / stride;
        const std::uint32_t j = static_cast<std::uint32_t>(x - node * stride);
        const std::uint32_t* block = src + node * (1 + cap);
        const std::uint32_t count = block[0];
        dst[x] = (j < count && j < cap) ? block[1 + j] : dev::kNoId;
    }
}

// FP32 rows -> BF16 rows (round to nearest even), rows of `out_row` elements, zero padded.
__global__ void to_bf16_kernel(const float* src, std::uint32_t src_row, __nv_bfloat16* dst,
                               std::uint32_t out_row, std::uint32_t n, std::uint32_t dim) {
    const std::size_t total = static_cast<std::size_t>(n) * out_row;
    for (std::size_t x = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; x < total;
         x += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
        const std::size_t r = x / out_row;
        const std::uint32_t e = static_cast<std::uint32_t>(x - r * out_row);
        dst[x] = __float2bfloat16_rn(e < dim ? src[r * src_row + e] : 0.0F);
    }
}

// FP32 rows -> FP8 E4M3 rows with one FP32 scale per row (max |x| / 448, stored in the row's
// last 4 bytes); one warp per row.
__global__ void to_fp8_kernel(const float* src, std::uint32_t src_row, unsigned char* dst,
                              std::uint32_t row_bytes, std::uint32_t n, std::uint32_t dim) {
    const int lane = threadIdx.x & 31;
    const std::size_t warp = (blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x) >> 5;
    const std::size_t warps = (static_cast<std::size_t>(gridDim.x) * blockDim.x) >> 5;
    for (std::size_t r = warp; r < n; r += warps) {
        const float* x = src + r * src_row;
        float m = 0.0F;
        for (std::uint32_t e = lane; e < dim; e += 32) {
            m = fmaxf(m, fabsf(x[e]));
        }
        for (int o = 16; o > 0; o >>= 1) {
            m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
        }
        const float scale = m > 0.0F ? m / 448.0F : 1.0F;
        unsigned char* row = dst + r * row_bytes;
        for (std::uint32_t e = lane; e < row_bytes - 4; e += 32) {
            const float v = e < dim ? x[e] / scale : 0.0F;
            row[e] = static_cast<unsigned char>(__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3));
        }
        if (lane == 0) {
            *reinterpret_cast<float*>(row + row_bytes - 4) = scale;
        }
    }
}

std::unique_ptr<DeviceGraph> upload_graph(const HnswIndex& index, int device, Precision precision) {
    gpu::use_device(device);
    auto dg = std::make_unique<DeviceGraph>();
    dg->device = device;
    const std::uint32_t n = static_cast<std::uint32_t>(index.size());
    const std::uint32_t dim = static_cast<std::uint32_t>(index.dim());
    const std::uint32_t M = static_cast<std::uint32_t>(index.params().M);
    if (index.size() >= (std::size_t{1} << 31)) {
        throw std::length_error("vdx: the GPU search holds at most 2^31 - 1 nodes");
    }
    if (M > 64) {
        throw std::invalid_argument("vdx: the GPU search supports M up to 64");
    }
    DeviceGraphView& v = dg->view;
    v.n = n;
    v.dim = dim;
    v.row32 = round_up(dim, 4);
    v.cap0 = 2 * M;
    v.stride0 = round_up(2 * M, 4);
    v.cap_up = M;
    v.stride_up = round_up(M, 4);
    v.max_level = static_cast<std::uint32_t>(index.max_level());
    v.entry = index.entry_point();
    v.metric = static_cast<std::uint32_t>(index.metric());
    v.precision = static_cast<std::uint32_t>(precision);
    cudaStream_t stream = gpu::workspace(device).stream;

    // FP32 rows, padded to 16 bytes.
    const std::size_t bytes32 = static_cast<std::size_t>(n) * v.row32 * 4;
    dg->vectors32_alloc = gpu::device_alloc(bytes32, "vectors");
    dg->bytes += bytes32;
    {
        std::vector<float> padded;
        const float* src = index.vectors().data();
        if (v.row32 != dim) {
            padded.assign(static_cast<std::size_t>(n) * v.row32, 0.0F);
            for (std::size_t r = 0; r < n; ++r) {
                std::memcpy(padded.data() + r * v.row32, src + r * dim, dim * 4);
            }
            src = padded.data();
        }
        gpu::check(cudaMemcpyAsync(dg->vectors32_alloc, src, bytes32, cudaMemcpyHostToDevice, stream),
                   "upload vectors");
        gpu::check(cudaStreamSynchronize(stream), "upload vectors");
    }
    v.vectors32 = static_cast<const float*>(dg->vectors32_alloc);
    if (precision == Precision::FP32) {
        v.vectors = v.vectors32;
        v.row_bytes = v.row32 * 4;
    } else if (precision == Precision::BF16) {
        const std::uint32_t row = round_up(dim, 8);
        v.row_bytes = row * 2;
        const std::size_t b = static_cast<std::size_t>(n) * v.row_bytes;
        dg->vectors_alloc = gpu::device_alloc(b, "bf16 vectors");
        dg->bytes += b;
        if (n > 0) {
            to_bf16_kernel<<<1184, 256, 0, stream>>>(v.vectors32, v.row32,
                                                     static_cast<__nv_bfloat16*>(dg->vectors_alloc), row, n, dim);
            gpu::check(cudaGetLastError(), "bf16 conversion");
        }
        v.vectors = dg->vectors_alloc;
    } else {
        v.row_bytes = round_up(dim + 4, 16);
        const std::size_t b = static_cast<std::size_t>(n) * v.row_bytes;
        dg->vectors_alloc = gpu::device_alloc(b, "fp8 vectors");
        dg->bytes += b;
        if (n > 0) {
            to_fp8_kernel<<<1184, 256, 0, stream>>>(v.vectors32, v.row32,
                                                    static_cast<unsigned char*>(dg->vectors_alloc),
                                                    v.row_bytes, n, dim);
            gpu::check(cudaGetLastError(), "fp8 conversion");
        }
        v.vectors = dg->vectors_alloc;
    }

    // Layer-0 links: upload the reference layout, repack on the device.
    {
        const std::size_t raw_bytes = static_cast<std::size_t>(n) * (1 + v.cap0) * 4;
        void* raw = gpu::device_alloc(raw_bytes, "raw links");
        gpu::check(cudaMemcpyAsync(raw, index.layer0().data(), raw_bytes, cudaMemcpyHostToDevice, stream),
                   "upload links");
        const std::size_t b = static_cast<std::size_t>(n) * v.stride0 * 4;
        dg->links0_alloc = gpu::device_alloc(b, "layer-0 links");
        dg->bytes += b;
        if (n > 0) {
            repack_links_kernel<<<1184, 256, 0, stream>>>(static_cast<const std::uint32_t*>(raw),
                                                          static_cast<std::uint32_t*>(dg->links0_alloc), n,
                                                          v.cap0, v.stride0);
            gpu::check(cudaGetLastError(), "repack links");
        }
        gpu::check(cudaStreamSynchronize(stream), "repack links");
        cudaFree(raw);
    }
    v.links0 = static_cast<const std::uint32_t*>(dg->links0_alloc);

    // Upper layers: per-node index of the first block, blocks repacked on the host (they are few).
    {
        std::vector<std::uint32_t> at(n, 0);
        std::vector<std::uint32_t> blocks;
        const auto levels = index.levels();
        std::uint32_t next = 0;
        for (std::uint32_t i = 0; i < n; ++i) {
            at[i] = next;
            const auto own = index.upper_blocks(i);
            for (std::uint32_t l = 0; l < levels[i]; ++l) {
                const std::uint32_t* b = own.data() + static_cast<std::size_t>(l) * (1 + M);
                for (std::uint32_t j = 0; j < v.stride_up; ++j) {
                    blocks.push_back(j < b[0] && j < M ? b[1 + j] : dev::kNoId);
                }
            }
            next += levels[i];
        }
        dg->upper_at_alloc = gpu::device_alloc(at.size() * 4, "upper index");
        dg->links_up_alloc = gpu::device_alloc(blocks.size() * 4, "upper links");
        dg->bytes += at.size() * 4 + blocks.size() * 4;
        gpu::check(cudaMemcpy(dg->upper_at_alloc, at.data(), at.size() * 4, cudaMemcpyHostToDevice),
                   "upload upper index");
        gpu::check(cudaMemcpy(dg->links_up_alloc, blocks.data(), blocks.size() * 4, cudaMemcpyHostToDevice),
                   "upload upper links");
    }
    v.upper_at = static_cast<const std::uint32_t*>(dg->upper_at_alloc);
    v.links_up = static_cast<const std::uint32_t*>(dg->links_up_alloc);
    gpu::attach_upper_copy(index, *dg, stream);
    return dg;
}

}  // namespace

const DeviceGraph& HnswIndex::device_graph(int device, Precision precision) const {
    if (!device_mutex_) {
        device_mutex_ = std::make_unique<std::mutex>();
    }
    const std::scoped_lock lock(*device_mutex_);
    const std::size_t slot = static_cast<std::size_t>(device) * 3 + static_cast<std::size_t>(precision);
    if (device_.size() <= slot) {
        device_.resize(slot + 1);
    }
    if (!device_[slot]) {
        device_[slot] = upload_graph(*this, device, precision);
    }
    return *device_[slot];
}

const DeviceGraph* HnswIndex::uploaded_graph(int device, Precision precision) const {
    if (!device_mutex_ || device < 0) {
        return nullptr;
    }
    const std::scoped_lock lock(*device_mutex_);
    const std::size_t slot = static_cast<std::size_t>(device) * 3 + static_cast<std::size_t>(precision);
    return slot < device_.size() ? device_[slot].get() : nullptr;
}

void HnswIndex::set_stop_model(StopModel model) {
    if (model.weights.size() != static_cast<std::size_t>(dev::kStopParams) ||
        model.mean.size() != static_cast<std::size_t>(dev::kStopFeatures) ||
        model.inv_std.size() != static_cast<std::size_t>(dev::kStopFeatures) ||
        model.proj.size() != 4 * dim()) {
        throw std::invalid_argument(std::format(
            "HnswIndex::set_stop_model: expected {} weights, 12 means, 12 scales and 4 x {} "
            "projections",
            dev::kStopParams, dim()));
    }
    if (!device_mutex_) {
        device_mutex_ = std::make_unique<std::mutex>();
    }
    const std::scoped_lock lock(*device_mutex_);
    stop_model_ = std::move(model);
    stop_net_.clear();
}

namespace {

const dev::DeviceStopNet& stop_net_for(const HnswIndex& ix, std::mutex& m,
                                       std::vector<std::shared_ptr<dev::DeviceStopNet>>& nets,
                                       int device, const char* where) {
    const std::scoped_lock lock(m);
    if (!ix.has_stop_model()) {
        throw std::invalid_argument(std::format("{}: learned_stop needs a model (set_stop_model)", where));
    }
    if (nets.size() <= static_cast<std::size_t>(device)) {
        nets.resize(device + 1);
    }
    if (!nets[device]) {
        const StopModel& sm = ix.stop_model();
        nets[device] = dev::upload_stop_net(sm.weights.data(), sm.mean.data(), sm.inv_std.data(),
                                            sm.proj.data(), static_cast<std::uint32_t>(ix.dim()),
                                            round_up(static_cast<std::uint32_t>(ix.dim()), 4), device);
    }
    return *nets[device];
}

}  // namespace

const dev::DeviceStopNet& HnswIndex::stop_net(int device) const {
    if (!device_mutex_) {
        device_mutex_ = std::make_unique<std::mutex>();
    }
    return stop_net_for(*this, *device_mutex_, stop_net_, device, "HnswIndex::search_batch");
}

void HnswIndex::search_batch_into(MatrixView<float> queries, std::size_t k, std::size_t ef,
                                  Id* ids, float* distances, std::uint32_t* counts,
                                  const SearchOptions& options, const char* where) const {
    detail::check_query_shape(where, {metric_, dim(), size()}, queries.dim(), k);
    const std::size_t nq = queries.rows();
    if (nq == 0) {
        return;
    }
    if (size() == 0) {
        std::fill(ids, ids + nq * k, dev::kNoId);
        std::fill(distances, distances + nq * k, std::numeric_limits<float>::infinity());
        std::fill(counts, counts + nq, 0U);
        return;
    }
    if (k > std::numeric_limits<std::uint32_t>::max() || ef > std::numeric_limits<std::uint32_t>::max()) {
        throw std::invalid_argument(std::format("{}: k and ef must fit in 32 bits", where));
    }
    const DeviceGraph& dg = device_graph(options.device, options.precision);
    gpu::Workspace& ws = gpu::workspace(options.device);
    ws.reserve(nq, dim(), k);
    // Page-locked queries are read by the kernel in place: each warp loads its query once, so
    // the 4·d bytes per query cross the bus while other warps search instead of in a copy ahead
    // of the launch. Pageable queries are copied first.
    const auto* in_place = static_cast<const float*>(gpu::mapped_host(queries.data().data()));
    if (in_place == nullptr) {
        gpu::check(cudaMemcpyAsync(ws.queries, queries.data().data(), queries.data().size_bytes(),
                                   cudaMemcpyHostToDevice, ws.stream),
                   "copy queries");
    }
    gpu::reset_small(ws);
    dev::SearchArgs a;
    a.g = dg.view;
    a.queries = in_place != nullptr ? in_place : ws.queries;
    a.nq = static_cast<std::uint32_t>(nq);
    a.qstride = static_cast<std::uint32_t>(dim());
    a.k = static_cast<std::uint32_t>(k);
    a.ef = static_cast<std::uint32_t>(ef);
    a.out_stride = static_cast<std::uint32_t>(k);
    // Page-locked result buffers are written by the kernel in place (it only stores to them),
    // so the results cross the bus as they are found; pageable ones are copied back after.
    auto* ids_in_place = static_cast<std::uint32_t*>(const_cast<void*>(gpu::mapped_host(ids)));
    auto* dists_in_place = static_cast<float*>(const_cast<void*>(gpu::mapped_host(distances)));
    auto* counts_in_place = static_cast<std::uint32_t*>(const_cast<void*>(gpu::mapped_host(counts)));
    a.out_ids = ids_in_place != nullptr ? ids_in_place : ws.ids;
    a.out_dists = dists_in_place != nullptr ? dists_in_place : ws.dists;
    a.out_counts = counts_in_place != nullptr ? counts_in_place : ws.counts;
    a.status = ws.small;
    a.claim = ws.small + 2;
    a.stats = reinterpret_cast<unsigned long long*>(ws.small + 16);
    a.rerank = rerank_width(options, k);
    if (options.learned_stop) {
        const dev::DeviceStopNet& net = stop_net_for(*this, *device_mutex_, stop_net_, options.device, where);
        a.stop = net.view;
        a.stop_enabled = &net;
        a.stop_threshold = options.stop_threshold;
        a.stop_gate = options.stop_gate;
    }
    const std::size_t ef_eff = std::min<std::size_t>(std::max(ef, k), size());
    dev::SearchPlan plan = dev::default_plan(dg.view, static_cast<std::uint32_t>(ef_eff), true);
    if (plan.global_slots > 0) {
        const std::uint32_t warps = dev::search_warps(a, plan);
        void* buf = ws.visited_for(plan.global_slots, warps);
        dev::bind_global_visited(a, plan, buf, ws.visited_stride, ws.visited_warps);
    }
    gpu::OrderScratch order(options.device, nq, ws.stream);
    a.entry_ids = order.entry_ids();
    a.entry_d = order.entry_d();
    a.order = order.order();
    gpu::check(dev::launch_search(a, plan, ws.stream), "search kernel");
    gpu::check(cudaMemcpyAsync(ws.small_host, ws.small, 256, cudaMemcpyDeviceToHost, ws.stream),
               "copy status");
    if (ids_in_place == nullptr) {
        gpu::check(cudaMemcpyAsync(ids, ws.ids, nq * k * 4, cudaMemcpyDeviceToHost, ws.stream), "copy ids");
    }
    if (dists_in_place == nullptr) {
        gpu::check(cudaMemcpyAsync(distances, ws.dists, nq * k * 4, cudaMemcpyDeviceToHost, ws.stream),
                   "copy distances");
    }
    if (counts_in_place == nullptr) {
        gpu::check(cudaMemcpyAsync(counts, ws.counts, nq * 4, cudaMemcpyDeviceToHost, ws.stream),
                   "copy counts");
    }
    gpu::check(cudaStreamSynchronize(ws.stream), "search");
    std::memcpy(ws.last_stats, ws.small_host + 16, sizeof ws.last_stats);
    gpu::raise_status(ws.small_host[0], where);
}

void HnswIndex::trace_search(MatrixView<float> queries, const Id* truth, std::size_t truth_k,
                             std::size_t k, std::size_t ef, const float* proj,
                             std::size_t max_points, float* features, std::uint8_t* hits,
                             std::uint32_t* points, std::uint8_t* final_hits, int device) const {
    const char* where = "HnswIndex::trace_search";
    detail::check_query_shape(where, {metric_, dim(), size()}, queries.dim(), k);
    if (k > 32 || truth_k > 32) {
        throw std::invalid_argument(std::format("{}: k and truth_k must be at most 32", where));
    }
    const std::size_t nq = queries.rows();
    if (nq == 0 || size() == 0) {
        std::fill(points, points + nq, 0U);
        std::fill(final_hits, final_hits + nq, std::uint8_t{0});
        return;
    }
    const DeviceGraph& dg = device_graph(device, Precision::FP32);
    gpu::Workspace& ws = gpu::workspace(device);
    ws.reserve(nq, dim(), k);
    const std::uint32_t row32 = round_up(static_cast<std::uint32_t>(dim()), 4);
    // Temporary trace buffers (training only, not the query path).
    struct Buffer {
        void* p = nullptr;
        Buffer(std::size_t bytes, const char* what) : p(gpu::device_alloc(bytes, what)) {}
        ~Buffer() { cudaFree(p); }
        Buffer(const Buffer&) = delete;
        Buffer& operator=(const Buffer&) = delete;
    };
    const std::size_t fbytes = nq * max_points * dev::kStopFeatures * 4;
    const Buffer dfeat(fbytes, "trace features");
    const Buffer dhits(nq * max_points, "trace hits");
    const Buffer dpoints(nq * 4, "trace points");
    const Buffer dfinal(nq, "trace final hits");
    const Buffer dtruth(nq * truth_k * 4, "trace truth");
    const Buffer dproj(4ull * row32 * 4, "trace projections");
    std::vector<float> proj_rows(4ull * row32, 0.0F);
    for (int i = 0; i < 4; ++i) {
        std::memcpy(proj_rows.data() + i * row32, proj + i * dim(), dim() * 4);
    }
    gpu::check(cudaMemcpyAsync(ws.queries, queries.data().data(), queries.data().size_bytes(),
                               cudaMemcpyHostToDevice, ws.stream), "copy queries");
    gpu::check(cudaMemcpyAsync(dtruth.p, truth, nq * truth_k * 4, cudaMemcpyHostToDevice, ws.stream),
               "copy truth");
    gpu::check(cudaMemcpyAsync(dproj.p, proj_rows.data(), proj_rows.size() * 4,
                               cudaMemcpyHostToDevice, ws.stream), "copy projections");
    gpu::reset_small(ws);
    dev::SearchArgs a;
    a.g = dg.view;
    a.queries = ws.queries;
    a.nq = static_cast<std::uint32_t>(nq);
    a.qstride = static_cast<std::uint32_t>(dim());
    a.k = static_cast<std::uint32_t>(k);
    a.ef = static_cast<std::uint32_t>(ef);
    a.out_stride = static_cast<std::uint32_t>(k);
    a.out_ids = ws.ids;
    a.out_dists = ws.dists;
    a.out_counts = ws.counts;
    a.status = ws.small;
    a.claim = ws.small + 2;
    a.stop.proj = static_cast<const float*>(dproj.p);
    a.trace = {static_cast<const std::uint32_t*>(dtruth.p), static_cast<std::uint32_t>(truth_k),
               static_cast<std::uint32_t>(max_points), static_cast<float*>(dfeat.p),
               static_cast<std::uint8_t*>(dhits.p), static_cast<std::uint32_t*>(dpoints.p),
               static_cast<std::uint8_t*>(dfinal.p)};
    const std::size_t ef_eff = std::min<std::size_t>(std::max(ef, k), size());
    dev::SearchPlan plan = dev::default_plan(dg.view, static_cast<std::uint32_t>(ef_eff));
    gpu::check(dev::launch_search(a, plan, ws.stream), "trace kernel");
    gpu::check(cudaMemcpyAsync(features, dfeat.p, fbytes, cudaMemcpyDeviceToHost, ws.stream), "copy features");
    gpu::check(cudaMemcpyAsync(hits, dhits.p, nq * max_points, cudaMemcpyDeviceToHost, ws.stream), "copy hits");
    gpu::check(cudaMemcpyAsync(points, dpoints.p, nq * 4, cudaMemcpyDeviceToHost, ws.stream), "copy points");
    gpu::check(cudaMemcpyAsync(final_hits, dfinal.p, nq, cudaMemcpyDeviceToHost, ws.stream), "copy final");
    gpu::check(cudaMemcpyAsync(ws.small_host, ws.small, 256, cudaMemcpyDeviceToHost, ws.stream), "status");
    gpu::check(cudaStreamSynchronize(ws.stream), "trace");
    gpu::raise_status(ws.small_host[0], where);
}

std::vector<std::vector<Neighbor>> HnswIndex::search_batch(MatrixView<float> queries, std::size_t k,
                                                           std::size_t ef, std::size_t) const {
    const std::size_t nq = queries.rows();
    std::vector<std::vector<Neighbor>> out(nq);
    if (nq == 0) {
        detail::check_query_shape("HnswIndex::search_batch", {metric_, dim(), size()}, queries.dim(), k);
        return out;
    }
    std::vector<Id> ids(nq * k);
    std::vector<float> d(nq * k);
    std::vector<std::uint32_t> c(nq);
    search_batch_into(queries, k, ef, ids.data(), d.data(), c.data());
    for (std::size_t q = 0; q < nq; ++q) {
        out[q].reserve(c[q]);
        for (std::uint32_t i = 0; i < c[q]; ++i) {
            out[q].push_back({d[q * k + i], ids[q * k + i]});
        }
    }
    return out;
}

std::vector<Neighbor> HnswIndex::search(std::span<const float> query, std::size_t k,
                                        std::size_t ef) const {
    detail::check_query("HnswIndex::search", {metric_, dim(), size()}, query, k);
    if (size() == 0) {
        return {};
    }
    std::vector<Id> ids(k);
    std::vector<float> d(k);
    std::uint32_t c = 0;
    search_batch_into(MatrixView<float>(query, dim()), k, ef, ids.data(), d.data(), &c, {},
                      "HnswIndex::search");
    std::vector<Neighbor> out;
    out.reserve(c);
    for (std::uint32_t i = 0; i < c; ++i) {
        out.push_back({d[i], ids[i]});
    }
    return out;
}

// ---------------------------------------------------------------------------------------------
// BruteForceIndex

BruteForceIndex::BruteForceIndex(std::size_t dim, Metric metric)
    : metric_(metric), vectors_(dim), device_mutex_(std::make_unique<std::mutex>()) {}
BruteForceIndex::~BruteForceIndex() = default;
BruteForceIndex::BruteForceIndex(BruteForceIndex&&) noexcept = default;
BruteForceIndex& BruteForceIndex::operator=(BruteForceIndex&&) noexcept = default;

void BruteForceIndex::store(std::span<const float> values) {
    if (!device_mutex_) {
        device_mutex_ = std::make_unique<std::mutex>();
    }
    {
        const std::scoped_lock lock(*device_mutex_);
        device_.clear();
    }
    const std::size_t first = size();
    vectors_.append(values);
    if (metric_ == Metric::Cosine) {
        for (std::size_t r = first; r < size(); ++r) {
            detail::normalize(vectors_.row(r));
        }
    }
}

Id BruteForceIndex::add(std::span<const float> vector) {
    detail::check_new_vectors("BruteForceIndex::add", {metric_, dim(), size()}, vector.size(), vector);
    const auto id = static_cast<Id>(size());
    store(vector);
    return id;
}

void BruteForceIndex::add(const Matrix<float>& vectors) { add(MatrixView<float>(vectors)); }

void BruteForceIndex::add(MatrixView<float> vectors) {
    detail::check_new_vectors("BruteForceIndex::add", {metric_, dim(), size()}, vectors.dim(),
                              vectors.data());
    store(vectors.data());
}

const DeviceBase& BruteForceIndex::device_base(int device) const {
    if (!device_mutex_) {
        device_mutex_ = std::make_unique<std::mutex>();
    }
    const std::scoped_lock lock(*device_mutex_);
    if (device_.size() <= static_cast<std::size_t>(device)) {
        device_.resize(device + 1);
    }
    if (!device_[device]) {
        gpu::use_device(device);
        auto b = std::make_unique<DeviceBase>();
        b->device = device;
        const std::uint32_t n = static_cast<std::uint32_t>(size());
        const std::uint32_t d = static_cast<std::uint32_t>(dim());
        const std::uint32_t row = round_up(d, 4);
        std::vector<float> padded(static_cast<std::size_t>(n) * row, 0.0F);
        for (std::size_t r = 0; r < n; ++r) {
            std::memcpy(padded.data() + r * row, vectors_.data().data() + r * d, d * 4);
        }
        b->alloc = gpu::device_alloc(padded.size() * 4, "brute-force vectors");
        gpu::check(cudaMemcpy(b->alloc, padded.data(), padded.size() * 4, cudaMemcpyHostToDevice),
                   "upload vectors");
        b->view = {static_cast<const float*>(b->alloc), n, d, row, static_cast<std::uint32_t>(metric_)};
        device_[device] = std::move(b);
    }
    return *device_[device];
}

void BruteForceIndex::search_batch_into(MatrixView<float> queries, std::size_t k, Id* ids,
                                        float* distances, std::uint32_t* counts, BruteMethod method,
                                        int device, const char* where) const {
    detail::check_query_shape(where, {metric_, dim(), size()}, queries.dim(), k);
    const std::size_t nq = queries.rows();
    if (nq == 0) {
        return;
    }
    if (size() == 0) {
        std::fill(ids, ids + nq * k, dev::kNoId);
        std::fill(distances, distances + nq * k, std::numeric_limits<float>::infinity());
        std::fill(counts, counts + nq, 0U);
        return;
    }
    const DeviceBase& b = device_base(device);
    gpu::Workspace& ws = gpu::workspace(device);
    ws.reserve(nq, dim(), k);
    gpu::check(cudaMemcpyAsync(ws.queries, queries.data().data(), queries.data().size_bytes(),
                               cudaMemcpyHostToDevice, ws.stream),
               "copy queries");
    gpu::reset_small(ws);
    dev::BruteArgs a;
    a.base = b.view;
    a.queries = ws.queries;
    a.nq = static_cast<std::uint32_t>(nq);
    a.qstride = static_cast<std::uint32_t>(dim());
    a.k = static_cast<std::uint32_t>(k);
    a.out_stride = static_cast<std::uint32_t>(k);
    a.out_ids = ws.ids;
    a.out_dists = ws.dists;
    a.out_counts = ws.counts;
    a.status = ws.small;
    if (method == BruteMethod::TensorCore) {
        {
            const std::scoped_lock lock(*device_mutex_);
            if (b.tc == nullptr) {
                gpu::check(dev::prepare_tc_base(b.view, ws.stream, &b.tc), "tensor-core preparation");
            }
        }
        void* work = ws.scratch_bytes(dev::bruteforce_tc_workspace(a.nq, b.view.n, b.view.dim, a.k));
        gpu::check(dev::launch_bruteforce_tc(a, *b.tc, work, ws.stream, ws.small + 8),
                   "brute-force (tensor cores)");
    } else {
        gpu::check(dev::launch_bruteforce_exact(a, ws.stream), "brute-force kernel");
    }
    gpu::check(cudaMemcpyAsync(ws.small_host, ws.small, 256, cudaMemcpyDeviceToHost, ws.stream),
               "copy status");
    gpu::check(cudaMemcpyAsync(ids, ws.ids, nq * k * 4, cudaMemcpyDeviceToHost, ws.stream), "copy ids");
    gpu::check(cudaMemcpyAsync(distances, ws.dists, nq * k * 4, cudaMemcpyDeviceToHost, ws.stream),
               "copy distances");
    gpu::check(cudaMemcpyAsync(counts, ws.counts, nq * 4, cudaMemcpyDeviceToHost, ws.stream), "copy counts");
    gpu::check(cudaStreamSynchronize(ws.stream), "brute force");
    std::fill(std::begin(ws.last_stats), std::end(ws.last_stats), 0ULL);
    ws.last_stats[0] = nq;
    ws.last_stats[12] = method == BruteMethod::TensorCore ? ws.small_host[8] : 0;
    gpu::raise_status(ws.small_host[0], where);
}

void BruteForceIndex::search_batch_device(const float* d_queries, std::size_t nq, std::size_t dim,
                                          std::size_t k, Id* d_ids, float* d_dists,
                                          std::uint32_t* d_counts, std::uint32_t* d_work,
                                          BruteMethod method, void* stream, int device) const {
    const char* where = "BruteForceIndex::search";
    detail::check_query_shape(where, {metric_, this->dim(), size()}, dim, k);
    auto s = static_cast<cudaStream_t>(stream);
    gpu::use_device(device);
    gpu::check(cudaMemsetAsync(d_work, 0, 64 * 4, s), "reset work words");
    gpu::check(cudaMemsetAsync(d_work + 1, 0xFF, 4, s), "reset work words");
    if (nq == 0) {
        return;
    }
    if (size() == 0) {
        gpu::check(cudaMemsetAsync(d_counts, 0, nq * 4, s), "clear counts");
        return;
    }
    const DeviceBase& b = device_base(device);
    dev::BruteArgs a;
    a.base = b.view;
    a.queries = d_queries;
    a.nq = static_cast<std::uint32_t>(nq);
    a.qstride = static_cast<std::uint32_t>(dim);
    a.k = static_cast<std::uint32_t>(k);
    a.out_stride = static_cast<std::uint32_t>(k);
    a.out_ids = d_ids;
    a.out_dists = d_dists;
    a.out_counts = d_counts;
    a.status = d_work;
    if (method == BruteMethod::TensorCore) {
        gpu::Workspace& ws = gpu::workspace(device);
        {
            const std::scoped_lock lock(*device_mutex_);
            if (b.tc == nullptr) {
                gpu::check(dev::prepare_tc_base(b.view, s, &b.tc), "tensor-core preparation");
            }
        }
        void* work = ws.scratch_bytes(dev::bruteforce_tc_workspace(a.nq, b.view.n, b.view.dim, a.k));
        gpu::check(dev::launch_bruteforce_tc(a, *b.tc, work, s, d_work + 8), "brute-force (tensor cores)");
    } else {
        gpu::check(dev::launch_bruteforce_exact(a, s), "brute-force kernel");
    }
}

std::vector<Neighbor> BruteForceIndex::search(std::span<const float> query, std::size_t k) const {
    detail::check_query("BruteForceIndex::search", {metric_, dim(), size()}, query, k);
    if (size() == 0) {
        return {};
    }
    std::vector<Id> ids(k);
    std::vector<float> d(k);
    std::uint32_t c = 0;
    search_batch_into(MatrixView<float>(query, dim()), k, ids.data(), d.data(), &c);
    std::vector<Neighbor> out;
    for (std::uint32_t i = 0; i < c; ++i) {
        out.push_back({d[i], ids[i]});
    }
    return out;
}

}  // namespace vdx
