#pragma once

// Per-thread device workspace and CUDA error plumbing shared by the host entry points.

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace vdx {
class HnswIndex;
struct DeviceGraph;
}  // namespace vdx

namespace vdx::gpu {

// A failed CUDA call, or no usable device (the C ABI maps it to VDX_ERR_CUDA).
struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& what) : std::runtime_error(what) {}
};

// A bounded device wait that gave up; the kernel released what it held (VDX_ERR_DEVICE_TIMEOUT).
struct DeviceTimeout : std::runtime_error {
    explicit DeviceTimeout(const std::string& what) : std::runtime_error(what) {}
};

// An out-of-range link id met in the device graph (VDX_ERR_DEVICE_BOUNDS).
struct DeviceBounds : std::runtime_error {
    explicit DeviceBounds(const std::string& what) : std::runtime_error(what) {}
};

// One host thread's buffers on one device: its stream, query and result buffers (grown on
// demand), 256 bytes of status / counter / statistics words and their pinned host copy.
// Layout of `small` (u32 words): [0] error code, [1] first failing row, [2] work counter,
// [3..7] spare, [8] uncertified count (tensor-core brute force), [16..] 64-bit statistics.
struct Workspace {
    int device = 0;
    cudaStream_t stream = nullptr;
    float* queries = nullptr;
    std::size_t queries_cap = 0;
    std::uint32_t* ids = nullptr;
    std::size_t ids_cap = 0;
    float* dists = nullptr;
    std::size_t dists_cap = 0;
    std::uint32_t* counts = nullptr;
    std::size_t counts_cap = 0;
    std::uint32_t* small = nullptr;
    std::uint32_t* small_host = nullptr;
    void* scratch = nullptr;
    std::size_t scratch_cap = 0;
    void* visited = nullptr;          // global visited tables of large-ef searches
    std::uint32_t visited_stride = 0; // slots per warp's table
    std::uint32_t visited_warps = 0;  // warps laid out
    unsigned long long last_stats[16] = {};

    Workspace() = default;
    Workspace(const Workspace&) = delete;
    Workspace& operator=(const Workspace&) = delete;
    ~Workspace();
    void reserve(std::size_t nq, std::size_t dim, std::size_t width);
    void* scratch_bytes(std::size_t bytes);
    // Global visited tables for `warps` warps of at least `slots` slots each. The layout only
    // grows (a larger stride or more warps re-lays it out and zeroes it on this workspace's
    // stream), so each warp's table and epoch counter keep their place between launches.
    void* visited_for(std::uint32_t slots, std::uint32_t warps);
};

// Scratch of an ordered search launch (three words per query: layer-0 entry ids, entry
// distances, claim order), allocated and freed in stream order from a per-device pool that keeps
// its memory, so launches on different streams never share it and nothing synchronizes.
class OrderScratch {
public:
    OrderScratch(int device, std::size_t nq, cudaStream_t stream);
    ~OrderScratch();
    OrderScratch(const OrderScratch&) = delete;
    OrderScratch& operator=(const OrderScratch&) = delete;
    std::uint32_t* entry_ids() const { return words_; }
    float* entry_d() const { return reinterpret_cast<float*>(words_ + nq_); }
    std::uint32_t* order() const { return words_ + 2 * nq_; }

private:
    std::uint32_t* words_ = nullptr;
    std::size_t nq_ = 0;
    cudaStream_t stream_ = nullptr;
};

void check(cudaError_t err, const char* what);
void use_device(int device);
void* device_alloc(std::size_t bytes, const char* what);
// The device address of page-locked host memory (cudaHostAlloc / cudaMallocHost / a mapped
// cudaHostRegister range), which kernels may read across the bus in place; nullptr for pageable
// memory or memory the device cannot address.
const void* mapped_host(const void* host);
Workspace& workspace(int device);
void reset_small(Workspace& ws);
void raise_status(std::uint32_t code, const char* where);

// Builds (or rebuilds) the device mirror's upper copy (vdx/device.hpp: the descent's blocks
// with their upper indices and the rows of nodes with upper layers, one allocation) from the
// mirror's current links and traversal rows, and sets the mirror's L2 access-policy window over
// it. Call after the mirror's upper layers or rows change.
void attach_upper_copy(const HnswIndex& index, DeviceGraph& dg, cudaStream_t stream);

}  // namespace vdx::gpu
