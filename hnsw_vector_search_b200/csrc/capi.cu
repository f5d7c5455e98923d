// The C ABI (include/vdx_b200.h): handles over the C++ host API, exceptions mapped to status
// codes with the message kept per thread.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <exception>
#include <format>
#include <new>
#include <stdexcept>
#include <string>

#include "../../include/vdx_b200.h"
#include "../host/src/internal.hpp"
#include "capi_internal.hpp"
#include "batcher.cuh"
#include "bruteforce.cuh"
#include "gpu_runtime.cuh"
#include "mlp.cuh"
#include "search.cuh"

namespace {

thread_local std::string g_error;

template <typename Fn>
vdx_status guarded(Fn&& fn) {
    try {
        fn();
        return VDX_OK;
    } catch (const std::invalid_argument& e) {
        g_error = e.what();
        return VDX_ERR_INVALID_ARGUMENT;
    } catch (const std::length_error& e) {
        g_error = e.what();
        return VDX_ERR_LENGTH;
    } catch (const vdx::gpu::CudaError& e) {
        g_error = e.what();
        return VDX_ERR_CUDA;
    } catch (const vdx::gpu::DeviceTimeout& e) {
        g_error = e.what();
        return VDX_ERR_DEVICE_TIMEOUT;
    } catch (const vdx::gpu::DeviceBounds& e) {
        g_error = e.what();
        return VDX_ERR_DEVICE_BOUNDS;
    } catch (const std::runtime_error& e) {
        g_error = e.what();
        return VDX_ERR_IO;
    } catch (const std::bad_alloc&) {
        g_error = "out of memory";
        return VDX_ERR_INTERNAL;
    } catch (const std::exception& e) {
        g_error = e.what();
        return VDX_ERR_INTERNAL;
    }
}

vdx::Metric metric_of(std::uint32_t code) {
    if (code > 2) {
        throw std::invalid_argument("unknown metric code");
    }
    return static_cast<vdx::Metric>(code);
}

vdx::SearchOptions options_of(const vdx_search_options* o) {
    vdx::SearchOptions s;
    if (o != nullptr) {
        if (o->precision > 2) {
            throw std::invalid_argument("unknown precision");
        }
        s.precision = static_cast<vdx::Precision>(o->precision);
        s.rerank = o->rerank;
        s.learned_stop = o->learned_stop != 0;
        s.stop_threshold = o->stop_threshold;
        if (o->stop_gate > 3) {
            throw std::invalid_argument("stop_gate must be at most 3");
        }
        s.stop_gate = o->stop_gate;
        s.device = o->device;
    }
    return s;
}

template <typename T>
void require(const T* p, const char* what) {
    if (p == nullptr) {
        throw std::invalid_argument(std::string(what) + " is NULL");
    }
}

}  // namespace

namespace vdx::capi {
void set_last_error(const std::string& message) { g_error = message; }
}  // namespace vdx::capi

extern "C" {

void vdx_testing_set_tc_wait_ns(uint64_t ns) { vdx::dev::set_tc_wait_ns(ns); }

const char* vdx_last_error(void) { return g_error.c_str(); }
const char* vdx_version(void) { return "vdx_b200 0.1.0 (sm_100a)"; }

int vdx_device_count(void) {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess ? n : 0;
}

vdx_status vdx_index_create(uint64_t dim, uint32_t metric, uint64_t M, uint64_t ef_construction,
                            uint64_t seed, vdx_index** out) {
    return guarded([&] {
        require(out, "out");
        *out = new vdx_index{vdx::HnswIndex(dim, metric_of(metric),
                                            {.M = M, .ef_construction = ef_construction, .seed = seed})};
    });
}

void vdx_index_free(vdx_index* index) { delete index; }

vdx_status vdx_index_add(vdx_index* index, const float* rows, uint64_t n, uint64_t dim,
                         uint64_t num_threads) {
    return guarded([&] {
        require(index, "index");
        if (n > 0) {
            require(rows, "rows");
        }
        index->index.add(vdx::MatrixView<float>(std::span<const float>(rows, n * dim), dim),
                         num_threads);
    });
}

vdx_status vdx_index_add_gpu(vdx_index* index, const float* rows, uint64_t n, uint64_t dim,
                             int32_t device) {
    return guarded([&] {
        require(index, "index");
        if (n > 0) {
            require(rows, "rows");
        }
        index->index.add_gpu(vdx::MatrixView<float>(std::span<const float>(rows, n * dim), dim), device);
    });
}

vdx_status vdx_index_add_one(vdx_index* index, const float* vector, uint64_t dim, uint32_t* id) {
    return guarded([&] {
        require(index, "index");
        require(vector, "vector");
        const vdx::Id got = index->index.add(std::span<const float>(vector, dim));
        if (id != nullptr) {
            *id = got;
        }
    });
}

vdx_status vdx_index_save(const vdx_index* index, const char* path) {
    return guarded([&] {
        require(index, "index");
        require(path, "path");
        index->index.save(path);
    });
}

vdx_status vdx_index_load(const char* path, vdx_index** out) {
    return guarded([&] {
        require(path, "path");
        require(out, "out");
        *out = new vdx_index{vdx::HnswIndex::load(path)};
    });
}

vdx_status vdx_index_save_device_image(const vdx_index* index, const char* path) {
    return guarded([&] {
        require(index, "index");
        require(path, "path");
        index->index.save_device_image(path);
    });
}

vdx_status vdx_index_load_device_image(const vdx_index* index, const char* path, int32_t device) {
    return guarded([&] {
        require(index, "index");
        require(path, "path");
        index->index.load_device_image(path, device);
    });
}

vdx_status vdx_index_graph_hash(const vdx_index* index, uint64_t* out) {
    return guarded([&] {
        require(index, "index");
        require(out, "out");
        *out = index->index.graph_hash();
    });
}

vdx_status vdx_index_info_get(const vdx_index* index, vdx_index_info* out) {
    return guarded([&] {
        require(index, "index");
        require(out, "out");
        const vdx::HnswIndex& i = index->index;
        *out = {i.size(),          i.dim(),         i.params().M,     i.params().ef_construction,
                i.params().seed,   i.max_level(),   i.entry_point(),  i.memory_bytes(),
                static_cast<uint32_t>(i.metric())};
    });
}

vdx_status vdx_index_inspect(const vdx_index* index, vdx_graph_report* out, char* first,
                             uint64_t cap) {
    return guarded([&] {
        require(index, "index");
        require(out, "out");
        const vdx::GraphReport r = index->index.inspect();
        *out = {r.violations.size(), r.reachable, r.max_level, r.mean_degree0};
        if (first != nullptr && cap > 0) {
            const std::string s = r.violations.empty() ? std::string() : r.violations.front();
            const std::size_t len = std::min<std::size_t>(s.size(), cap - 1);
            std::memcpy(first, s.data(), len);
            first[len] = '\0';
        }
    });
}

vdx_status vdx_search_batch(const vdx_index* index, const float* queries, uint64_t nq,
                            uint64_t dim, uint64_t k, uint64_t ef, uint32_t* ids, float* dists,
                            uint32_t* counts, const vdx_search_options* opts) {
    return guarded([&] {
        require(index, "index");
        if (nq > 0) {
            require(queries, "queries");
            require(ids, "ids");
            require(dists, "dists");
            require(counts, "counts");
        }
        if (dim == 0) {
            throw std::invalid_argument("HnswIndex::search_batch: query has dimension 0, index has " +
                                        std::to_string(index->index.dim()));
        }
        index->index.search_batch_into(
            vdx::MatrixView<float>(std::span<const float>(queries, nq * dim), dim), k, ef, ids,
            dists, counts, options_of(opts));
    });
}

vdx_status vdx_search(const vdx_index* index, const float* query, uint64_t dim, uint64_t k,
                      uint64_t ef, uint32_t* ids, float* dists, uint32_t* count) {
    return guarded([&] {
        require(index, "index");
        require(query, "query");
        require(count, "count");
        const auto found = index->index.search(std::span<const float>(query, dim), k, ef);
        for (std::size_t i = 0; i < k; ++i) {
            ids[i] = i < found.size() ? found[i].id : 0xFFFFFFFFu;
            dists[i] = i < found.size() ? found[i].distance : __builtin_inff();
        }
        *count = static_cast<uint32_t>(found.size());
    });
}

vdx_status vdx_last_stats(uint64_t* out, uint64_t count) {
    return guarded([&] {
        require(out, "out");
        int device = 0;
        cudaGetDevice(&device);
        const vdx::gpu::Workspace& ws = vdx::gpu::workspace(device);
        for (uint64_t i = 0; i < count && i < 16; ++i) {
            out[i] = ws.last_stats[i];
        }
    });
}

vdx_status vdx_index_upload(const vdx_index* index, int32_t device, uint32_t precision) {
    return guarded([&] {
        require(index, "index");
        if (precision > 2) {
            throw std::invalid_argument("unknown precision");
        }
        if (index->index.size() > 0) {
            (void)index->index.device_graph(device, static_cast<vdx::Precision>(precision));
        }
    });
}

uint64_t vdx_work_words(void) { return 64; }

uint32_t vdx_search_kernels_last(void) { return static_cast<uint32_t>(vdx::dev::search_kernels_per_launch()); }

vdx_status vdx_search_batch_device(const vdx_index* index, const float* d_queries, uint64_t nq,
                                   uint64_t dim, const uint32_t* d_k, const uint32_t* d_ef,
                                   uint32_t k_uniform, uint32_t ef_uniform, uint32_t out_stride,
                                   uint32_t* d_ids, float* d_dists, uint32_t* d_counts,
                                   uint32_t* d_work, const vdx_search_options* opts,
                                   void* stream) {
    return guarded([&] {
        require(index, "index");
        require(d_work, "d_work");
        const vdx::HnswIndex& h = index->index;
        const vdx::SearchOptions o = options_of(opts);
        vdx::detail::check_query_shape("HnswIndex::search_batch", {h.metric(), h.dim(), h.size()},
                                       dim, d_k == nullptr ? k_uniform : 1);
        if (nq > 0) {
            require(d_queries, "d_queries");
            require(d_ids, "d_ids");
            require(d_dists, "d_dists");
            require(d_counts, "d_counts");
            if (d_k == nullptr && out_stride < k_uniform) {
                throw std::invalid_argument("vdx_search_batch_device: out_stride is smaller than k");
            }
        }
        auto s = static_cast<cudaStream_t>(stream);
        vdx::gpu::use_device(o.device);
        vdx::gpu::check(cudaMemsetAsync(d_work, 0, vdx_work_words() * 4, s), "reset work words");
        vdx::gpu::check(cudaMemsetAsync(d_work + 1, 0xFF, 4, s), "reset work words");
        if (nq == 0 || h.size() == 0) {
            if (nq > 0) {
                vdx::gpu::check(cudaMemsetAsync(d_counts, 0, nq * 4, s), "clear counts");
            }
            return;
        }
        const vdx::DeviceGraph& g = h.device_graph(o.device, o.precision);
        vdx::dev::SearchArgs a;
        a.g = g.view;
        a.queries = d_queries;
        a.nq = static_cast<uint32_t>(nq);
        a.qstride = static_cast<uint32_t>(dim);
        a.k_per_q = d_k;
        a.ef_per_q = d_ef;
        a.k = k_uniform;
        a.ef = ef_uniform;
        a.out_stride = out_stride;
        a.out_ids = d_ids;
        a.out_dists = d_dists;
        a.out_counts = d_counts;
        a.status = d_work;
        a.claim = d_work + 2;
        a.stats = reinterpret_cast<unsigned long long*>(d_work + 16);
        const uint32_t kk = std::max<uint32_t>(k_uniform, 1);
        a.rerank = vdx::rerank_width(o, kk);
        if (o.learned_stop) {
            const vdx::dev::DeviceStopNet& net = h.stop_net(o.device);
            a.stop = net.view;
            a.stop_enabled = &net;
            a.stop_threshold = o.stop_threshold;
            a.stop_gate = o.stop_gate;
        }
        // Per-query ef: the capacity must cover the largest; the caller's uniform ef bounds it.
        const uint64_t cap = std::min<uint64_t>(std::max<uint64_t>(ef_uniform, kk), h.size());
        const vdx::dev::SearchPlan plan = vdx::dev::default_plan(g.view, static_cast<uint32_t>(cap));
        const vdx::gpu::OrderScratch order(o.device, nq, s);
        a.entry_ids = order.entry_ids();
        a.entry_d = order.entry_d();
        a.order = order.order();
        vdx::gpu::check(vdx::dev::launch_search(a, plan, s), "search kernel");
    });
}

struct vdx_batcher {
    vdx::dev::Batcher b;
};

namespace {
void check_batch_size(const vdx_batcher& b, uint64_t nq) {
    if (nq > b.b.max_queries) {
        throw std::invalid_argument(
            std::format("vdx_batcher: batch of {} exceeds the maximum {}", nq, b.b.max_queries));
    }
}
}  // namespace

vdx_status vdx_batcher_create(const vdx_index* index, int32_t device, uint32_t precision,
                              uint32_t max_queries, uint32_t max_k, uint32_t max_ef,
                              vdx_batcher** out) {
    return guarded([&] {
        require(index, "index");
        require(out, "out");
        if (precision > 2) {
            throw std::invalid_argument("unknown precision");
        }
        *out = new vdx_batcher{vdx::dev::Batcher(index->index, device,
                                                 static_cast<vdx::Precision>(precision), max_queries,
                                                 max_k, max_ef)};
    });
}

void vdx_batcher_free(vdx_batcher* batcher) { delete batcher; }

vdx_status vdx_batcher_run(vdx_batcher* batcher, const float* queries, uint64_t nq,
                           const uint32_t* k_per_q, const uint32_t* ef_per_q, uint32_t* ids,
                           float* dists, uint32_t* counts) {
    return guarded([&] {
        require(batcher, "batcher");
        if (nq == 0) {
            return;
        }
        check_batch_size(*batcher, nq);
        batcher->b.run(queries, static_cast<uint32_t>(nq), k_per_q, ef_per_q, ids, dists, counts);
    });
}

vdx_status vdx_batcher_submit(vdx_batcher* batcher, const float* queries, uint64_t nq,
                              const uint32_t* k_per_q, const uint32_t* ef_per_q) {
    return guarded([&] {
        require(batcher, "batcher");
        check_batch_size(*batcher, nq);
        batcher->b.submit(queries, static_cast<uint32_t>(nq), k_per_q, ef_per_q);
    });
}

vdx_status vdx_batcher_wait(vdx_batcher* batcher, uint32_t* ids, float* dists, uint32_t* counts) {
    return guarded([&] {
        require(batcher, "batcher");
        batcher->b.wait(ids, dists, counts);
    });
}

vdx_status vdx_batcher_autotune(vdx_batcher* batcher, const float* queries, uint64_t nq,
                                const uint32_t* k_per_q, const uint32_t* ef_per_q,
                                vdx_plan_timing* timings, uint64_t cap, uint64_t* n_out) {
    return guarded([&] {
        require(batcher, "batcher");
        check_batch_size(*batcher, nq);
        const auto tried = batcher->b.autotune(queries, static_cast<uint32_t>(nq), k_per_q, ef_per_q);
        for (std::size_t i = 0; i < tried.size() && i < cap; ++i) {
            const vdx::dev::SearchPlan& pl = tried[i].plan;
            timings[i] = {tried[i].ef_class, pl.warps_per_block, pl.rows_cap,
                          pl.global_slots > 0 ? 0u : pl.hash_slots, pl.efcap, tried[i].ms,
                          pl.global_slots};
        }
        if (n_out != nullptr) {
            *n_out = tried.size();
        }
    });
}

vdx_status vdx_index_set_stop_model(vdx_index* index, const float* weights, const float* mean,
                                    const float* inv_std, const float* proj) {
    return guarded([&] {
        require(index, "index");
        require(weights, "weights");
        require(mean, "mean");
        require(inv_std, "inv_std");
        require(proj, "proj");
        const std::size_t dim = index->index.dim();
        vdx::StopModel m;
        m.weights.assign(weights, weights + vdx::dev::kStopParams);
        m.mean.assign(mean, mean + vdx::dev::kStopFeatures);
        m.inv_std.assign(inv_std, inv_std + vdx::dev::kStopFeatures);
        m.proj.assign(proj, proj + 4 * dim);
        index->index.set_stop_model(std::move(m));
    });
}

vdx_status vdx_stop_trace(const vdx_index* index, const float* queries, uint64_t nq, uint64_t dim,
                          const uint32_t* truth, uint64_t truth_k, uint64_t k, uint64_t ef,
                          const float* proj, uint64_t max_points, float* features, uint8_t* hits,
                          uint32_t* points, uint8_t* final_hits, int32_t device) {
    return guarded([&] {
        require(index, "index");
        require(proj, "proj");
        if (nq > 0) {
            require(queries, "queries");
            require(truth, "truth");
        }
        index->index.trace_search(
            vdx::MatrixView<float>(std::span<const float>(queries, nq * dim), dim == 0 ? 1 : dim),
            truth, truth_k, k, ef, proj, max_points, features, hits, points, final_hits, device);
    });
}

vdx_status vdx_mlp_train(const float* x, const float* y, uint64_t n, uint32_t epochs, uint64_t batch,
                         float lr, uint64_t seed, float* weights, float* mean, float* inv_std,
                         float* loss_per_epoch) {
    return guarded([&] {
        require(x, "x");
        require(y, "y");
        require(weights, "weights");
        vdx::dev::MlpTrainConfig cfg;
        cfg.epochs = static_cast<int>(epochs);
        cfg.batch = batch;
        cfg.lr = lr;
        cfg.seed = seed;
        vdx::gpu::use_device(0);
        vdx::dev::mlp_train(x, y, n, cfg, weights, mean, inv_std, loss_per_epoch);
    });
}

vdx_status vdx_mlp_gradient(const float* x, const float* y, uint64_t n, const float* weights,
                            float* grad, float* loss) {
    return guarded([&] {
        require(x, "x");
        require(weights, "weights");
        require(grad, "grad");
        vdx::gpu::use_device(0);
        vdx::dev::mlp_gradient(x, y, n, weights, grad, loss);
    });
}

vdx_status vdx_mlp_probabilities(const float* x, uint64_t n, const float* weights, const float* mean,
                                 const float* inv_std, float* prob) {
    return guarded([&] {
        require(x, "x");
        require(weights, "weights");
        vdx::gpu::use_device(0);
        vdx::dev::mlp_probabilities(x, n, weights, mean, inv_std, prob);
    });
}

vdx_status vdx_bf_create(uint64_t dim, uint32_t metric, vdx_bruteforce** out) {
    return guarded([&] {
        require(out, "out");
        *out = new vdx_bruteforce{vdx::BruteForceIndex(dim, metric_of(metric))};
    });
}

void vdx_bf_free(vdx_bruteforce* index) { delete index; }

vdx_status vdx_bf_add(vdx_bruteforce* index, const float* rows, uint64_t n, uint64_t dim) {
    return guarded([&] {
        require(index, "index");
        if (n > 0) {
            require(rows, "rows");
        }
        index->index.add(vdx::MatrixView<float>(std::span<const float>(rows, n * dim), dim));
    });
}

uint64_t vdx_bf_size(const vdx_bruteforce* index) { return index == nullptr ? 0 : index->index.size(); }

vdx_status vdx_bf_search_batch(const vdx_bruteforce* index, const float* queries, uint64_t nq,
                               uint64_t dim, uint64_t k, uint32_t method, uint32_t* ids,
                               float* dists, uint32_t* counts) {
    return guarded([&] {
        require(index, "index");
        if (method > 1) {
            throw std::invalid_argument("unknown brute-force method");
        }
        if (dim == 0) {
            throw std::invalid_argument("BruteForceIndex::search: query has dimension 0");
        }
        index->index.search_batch_into(
            vdx::MatrixView<float>(std::span<const float>(queries, nq * dim), dim), k, ids, dists,
            counts, static_cast<vdx::BruteMethod>(method));
    });
}

vdx_status vdx_bf_search_batch_device(const vdx_bruteforce* index, const float* d_queries,
                                      uint64_t nq, uint64_t dim, uint64_t k, uint32_t method,
                                      uint32_t* d_ids, float* d_dists, uint32_t* d_counts,
                                      uint32_t* d_work, void* stream) {
    return guarded([&] {
        require(index, "index");
        require(d_work, "d_work");
        if (method > 1) {
            throw std::invalid_argument("unknown brute-force method");
        }
        index->index.search_batch_device(d_queries, nq, dim, k, d_ids, d_dists, d_counts, d_work,
                                         static_cast<vdx::BruteMethod>(method), stream);
    });
}

float vdx_host_l2(const float* a, const float* b, uint64_t dim) {
    return vdx::detail::l2_squared_raw(a, b, dim);
}
float vdx_host_ip(const float* a, const float* b, uint64_t dim) {
    return vdx::detail::inner_product_raw(a, b, dim);
}
uint64_t vdx_xxh64(const void* data, uint64_t size, uint64_t seed) {
    return vdx::detail::xxh64(data, size, seed);
}

}  // extern "C"
