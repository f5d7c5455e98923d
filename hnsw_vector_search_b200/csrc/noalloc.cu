// vdx_search_batch_device_noalloc: the device-buffer HNSW search for callers that cannot
// allocate device memory.
//
// Who needs it: code that runs where device allocation is not available or not allowed, e.g. a
// host process whose device memory is handed out by an external pool manager (inference
// servers that pre-reserve all of HBM), a real-time path that must not call cudaMalloc (it can
// block and synchronize the device), or a plugin that may only use the buffers its host passes
// in. vdx_search_batch_device needs a caller-provided work buffer (d_work); this variant keeps
// that launch state in a file-scope __device__ array instead, so the caller passes only its
// queries and result buffers, and the call allocates nothing.
//
// The static array holds the search launch's work words: the error code, the first failing row,
// the query-claim counter and the statistics words (kStaticWorkWords u32 = 256 bytes, the same
// layout as d_work). Every GPU that loads this library holds these 256 bytes until the process
// exits. All calls on a device share the one array: each call clears it before its launch, and
// two calls whose kernels overlap on the GPU (different streams, or threads) race on it and may
// return wrong results or errors; callers must serialize them.
//
// Set-up: the first call on each device looks up the array's device address with
// cudaGetSymbolAddress (in host code the array's name is only a host-side stand-in, not a device
// address) and keeps it; make that first call before any stream capture begins. The address is
// kept for the life of the process: a cudaDeviceReset (or any teardown of the primary context)
// after that first call is not supported, since the kept address would then be stale.
//
// The learned stop is not offered here: its network lives in device memory that the index
// allocates on first use, so a call asking for it is rejected (VDX_ERR_INVALID_ARGUMENT)
// rather than silently running the plain search.

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/vdx_b200.h"
#include "../host/src/internal.hpp"
#include "capi_internal.hpp"
#include "gpu_runtime.cuh"
#include "search.cuh"

namespace {

constexpr std::uint32_t kStaticWorkWords = 64;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) std::uint32_t g_static_work[kStaticWorkWords];

std::mutex g_setup;
std::uint32_t* g_work_address[kMaxDevices] = {};

// The device address of g_static_work on the current device, looked up once per device.
std::uint32_t* static_work(int device) {
    if (device < 0 || device >= kMaxDevices) {
        throw std::invalid_argument("vdx_search_batch_device_noalloc: device index out of range");
    }
    const std::scoped_lock lock(g_setup);
    if (g_work_address[device] == nullptr) {
        void* p = nullptr;
        vdx::gpu::check(cudaGetSymbolAddress(&p, g_static_work), "cudaGetSymbolAddress");
        g_work_address[device] = static_cast<std::uint32_t*>(p);
    }
    return g_work_address[device];
}

}  // namespace

extern "C" vdx_status vdx_search_batch_device_noalloc(
    const vdx_index* index, const float* d_queries, uint64_t nq, uint64_t dim,
    const uint32_t* d_k, const uint32_t* d_ef, uint32_t k_uniform, uint32_t ef_uniform,
    uint32_t out_stride, uint32_t* d_ids, float* d_dists, uint32_t* d_counts,
    const vdx_search_options* opts, void* stream) {
    try {
        if (index == nullptr) {
            throw std::invalid_argument("vdx_search_batch_device_noalloc: index is NULL");
        }
        const vdx::HnswIndex& h = index->index;
        vdx::SearchOptions o;
        if (opts != nullptr) {
            if (opts->precision > 2) {
                throw std::invalid_argument("unknown precision");
            }
            if (opts->learned_stop != 0) {
                throw std::invalid_argument(
                    "vdx_search_batch_device_noalloc: the learned stop is not available without "
                    "allocation; use vdx_search_batch_device");
            }
            o.precision = static_cast<vdx::Precision>(opts->precision);
            o.rerank = opts->rerank;
            o.device = opts->device;
        }
        const char* where = "HnswIndex::search_batch";
        vdx::detail::check_query_shape(where, {h.metric(), h.dim(), h.size()}, dim,
                                       d_k == nullptr ? k_uniform : 1);
        if (nq > 0) {
            const auto require = [](const void* p, const char* what) {
                if (p == nullptr) {
                    throw std::invalid_argument(std::string("vdx_search_batch_device_noalloc: ") +
                                                what + " is NULL");
                }
            };
            require(d_queries, "d_queries");
            require(d_ids, "d_ids");
            require(d_dists, "d_dists");
            require(d_counts, "d_counts");
            if (d_k == nullptr && out_stride < k_uniform) {
                throw std::invalid_argument(
                    "vdx_search_batch_device_noalloc: out_stride is smaller than k");
            }
        }
        if (vdx_work_words() > kStaticWorkWords) {
            throw std::length_error(
                "vdx_search_batch_device_noalloc: the launch needs " +
                std::to_string(vdx_work_words()) + " work words, the static scratch holds " +
                std::to_string(kStaticWorkWords));
        }
        vdx::gpu::use_device(o.device);
        std::uint32_t* work = static_work(o.device);
        auto s = static_cast<cudaStream_t>(stream);
        vdx::gpu::check(cudaMemsetAsync(work, 0, kStaticWorkWords * 4, s), "clear static scratch");
        vdx::gpu::check(cudaMemsetAsync(work + 1, 0xFF, 4, s), "clear static scratch");
        if (nq == 0 || h.size() == 0) {
            if (nq > 0) {
                vdx::gpu::check(cudaMemsetAsync(d_counts, 0, nq * 4, s), "clear counts");
            }
            vdx::gpu::check(cudaStreamSynchronize(s), "search");
            return VDX_OK;
        }
        const vdx::DeviceGraph* g = h.uploaded_graph(o.device, o.precision);
        if (g == nullptr) {
            throw std::invalid_argument(
                "vdx_search_batch_device_noalloc: the index has no device copy for this device "
                "and precision; call vdx_index_upload first (it allocates, this call does not)");
        }
        vdx::dev::SearchArgs a;
        a.g = g->view;
        a.queries = d_queries;
        a.nq = static_cast<std::uint32_t>(nq);
        a.qstride = static_cast<std::uint32_t>(dim);
        a.k_per_q = d_k;
        a.ef_per_q = d_ef;
        a.k = k_uniform;
        a.ef = ef_uniform;
        a.out_stride = out_stride;
        a.out_ids = d_ids;
        a.out_dists = d_dists;
        a.out_counts = d_counts;
        a.status = work;
        a.claim = work + 2;
        a.stats = reinterpret_cast<unsigned long long*>(work + 16);
        const std::uint32_t kk = k_uniform > 0 ? k_uniform : 1;
        a.rerank = vdx::rerank_width(o, kk);
        const std::uint64_t ef_cap = ef_uniform > kk ? ef_uniform : kk;
        const std::uint64_t cap = ef_cap < h.size() ? ef_cap : h.size();
        const vdx::dev::SearchPlan plan = vdx::dev::default_plan(g->view, static_cast<std::uint32_t>(cap));
        vdx::gpu::check(vdx::dev::launch_search(a, plan, s), "search kernel");
        std::uint32_t status[2] = {0, 0};
        vdx::gpu::check(cudaMemcpyAsync(status, work, sizeof status, cudaMemcpyDeviceToHost, s),
                        "read status");
        vdx::gpu::check(cudaStreamSynchronize(s), "search");
        vdx::gpu::raise_status(status[0], where);
        return VDX_OK;
    } catch (const std::invalid_argument& e) {
        vdx::capi::set_last_error(e.what());
        return VDX_ERR_INVALID_ARGUMENT;
    } catch (const std::length_error& e) {
        vdx::capi::set_last_error(e.what());
        return VDX_ERR_LENGTH;
    } catch (const vdx::gpu::CudaError& e) {
        vdx::capi::set_last_error(e.what());
        return VDX_ERR_CUDA;
    } catch (const vdx::gpu::DeviceTimeout& e) {
        vdx::capi::set_last_error(e.what());
        return VDX_ERR_DEVICE_TIMEOUT;
    } catch (const vdx::gpu::DeviceBounds& e) {
        vdx::capi::set_last_error(e.what());
        return VDX_ERR_DEVICE_BOUNDS;
    } catch (const std::exception& e) {
        vdx::capi::set_last_error(e.what());
        return VDX_ERR_INTERNAL;
    }
}
