// Uneven batches through one captured launch graph.
//
// A request stream mixes batch sizes (1 .. thousands of queries), k and ef. The search kernel
// already reads each query's k and ef, and the batch size, from device memory, so one captured
// launch serves any batch up to a fixed capacity. What a single launch cannot do well is mix a
// query at ef = 600 with queries at ef = 20: its shared-memory plan (result-list capacity,
// visited-filter slots) is sized for the largest ef, which cuts the resident warps for every
// query. So the Batcher splits each batch into ef classes (effective ef <= 64, <= 256, <= 1024,
// ... up to the largest ef it accepts), each with its own plan and fixed device / pinned
// buffers. The graph holds one branch per class (work-word reset + persistent search kernel);
// the branches run concurrently, so one class's blocks fill the SMs another class's tail
// leaves idle. Within a class the rows are staged longest-first (descending ef), the classic
// longest-processing-time order, so the persistent warps that claim rows in order finish
// together.
//
// Per batch the host stages the rows (pinned), issues one copy per class buffer, replays the
// graph and copies the results back; results return in the caller's row order. The autotuner
// times candidate plans (warps per block, rows per gather round, visited-filter slots) for each
// class on a sample batch with CUDA events and keeps each class's fastest.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <format>
#include <numeric>
#include <stdexcept>
#include <vector>

#include "batcher.cuh"
#include "gpu_runtime.cuh"
#include "search.cuh"
#include "vdx/device.hpp"

namespace vdx::dev {

namespace {

template <typename T>
T* dalloc(std::size_t n, const char* what) {
    void* p = gpu::device_alloc(std::max<std::size_t>(n, 1) * sizeof(T), what);
    gpu::check(cudaMemset(p, 0, std::max<std::size_t>(n, 1) * sizeof(T)), what);
    return static_cast<T*>(p);
}
template <typename T>
T* halloc(std::size_t n) {
    void* p = nullptr;
    gpu::check(cudaMallocHost(&p, std::max<std::size_t>(n, 1) * sizeof(T)), "cudaMallocHost");
    std::memset(p, 0, std::max<std::size_t>(n, 1) * sizeof(T));
    return static_cast<T*>(p);
}

constexpr std::uint32_t kWorkWords = 64;
constexpr std::uint32_t kRerankPerK = 4;

}  // namespace

Batcher::Batcher(const HnswIndex& idx, int dev, Precision prec, std::uint32_t max_q,
                 std::uint32_t max_k_, std::uint32_t max_ef_)
    : index(idx), device(dev), precision(prec), max_queries(max_q), max_k(max_k_), max_ef(max_ef_) {
    if (max_q == 0 || max_k_ == 0) {
        throw std::invalid_argument("Batcher: max_queries and max_k must be positive");
    }
    if (index.size() == 0) {
        throw std::invalid_argument("Batcher: the index is empty");
    }
    gpu::use_device(device);
    index_size = index.size();
    graph_view = index.device_graph(device, precision).view;
    dim = static_cast<std::uint32_t>(index.dim());
    gpu::check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
    gpu::check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");

    const std::uint32_t n = static_cast<std::uint32_t>(std::min<std::size_t>(index_size, 0xFFFFFFFFu));
    const std::uint32_t top = std::max<std::uint32_t>(1, std::min(std::max(max_ef, max_k), n));
    std::vector<std::uint32_t> caps;
    for (std::uint32_t c = 64; c < top; c *= 4) {
        caps.push_back(c);
    }
    caps.push_back(top);
    classes.resize(caps.size());
    joins.resize(caps.size());
    const std::size_t rows_q = static_cast<std::size_t>(max_q) * dim;
    const std::size_t rows_out = static_cast<std::size_t>(max_q) * max_k;
    for (std::size_t i = 0; i < caps.size(); ++i) {
        EfClass& c = classes[i];
        c.cap = caps[i];
        c.plan = default_plan(graph_view, c.cap, true);
        gpu::check(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "stream");
        gpu::check(cudaEventCreateWithFlags(&joins[i], cudaEventDisableTiming), "event");
        c.d_queries = dalloc<float>(rows_q, "batch queries");
        c.d_k = dalloc<std::uint32_t>(max_q, "batch k");
        c.d_ef = dalloc<std::uint32_t>(max_q, "batch ef");
        c.d_nq = dalloc<std::uint32_t>(1, "batch size");
        c.d_ids = dalloc<std::uint32_t>(rows_out, "batch ids");
        c.d_dists = dalloc<float>(rows_out, "batch distances");
        c.d_counts = dalloc<std::uint32_t>(max_q, "batch counts");
        c.d_work = dalloc<std::uint32_t>(kWorkWords, "batch work words");
        c.d_order = dalloc<std::uint32_t>(3 * static_cast<std::size_t>(max_q), "batch order");
        c.h_queries = halloc<float>(rows_q);
        c.h_k = halloc<std::uint32_t>(max_q);
        c.h_ef = halloc<std::uint32_t>(max_q);
        c.h_nq = halloc<std::uint32_t>(1);
        c.h_ids = halloc<std::uint32_t>(rows_out);
        c.h_dists = halloc<float>(rows_out);
        c.h_counts = halloc<std::uint32_t>(max_q);
        c.h_work = halloc<std::uint32_t>(kWorkWords);
    }
    capture();
}

Batcher::~Batcher() {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (stream != nullptr) {
        cudaStreamSynchronize(stream);
    }
    if (exec != nullptr) {
        cudaGraphExecDestroy(exec);
    }
    if (graph != nullptr) {
        cudaGraphDestroy(graph);
    }
    for (EfClass& c : classes) {
        if (c.stream != nullptr) {
            cudaStreamSynchronize(c.stream);
            cudaStreamDestroy(c.stream);
        }
        for (void* p : {static_cast<void*>(c.d_queries), static_cast<void*>(c.d_k),
                        static_cast<void*>(c.d_ef), static_cast<void*>(c.d_nq),
                        static_cast<void*>(c.d_ids), static_cast<void*>(c.d_dists),
                        static_cast<void*>(c.d_counts), static_cast<void*>(c.d_work), static_cast<void*>(c.d_order), c.d_visited}) {
            cudaFree(p);
        }
        for (void* p : {static_cast<void*>(c.h_queries), static_cast<void*>(c.h_k),
                        static_cast<void*>(c.h_ef), static_cast<void*>(c.h_nq),
                        static_cast<void*>(c.h_ids), static_cast<void*>(c.h_dists),
                        static_cast<void*>(c.h_counts), static_cast<void*>(c.h_work)}) {
            cudaFreeHost(p);
        }
    }
    for (cudaEvent_t e : joins) {
        if (e != nullptr) {
            cudaEventDestroy(e);
        }
    }
    if (fork != nullptr) {
        cudaEventDestroy(fork);
    }
    if (stream != nullptr) {
        cudaStreamDestroy(stream);
    }
    cudaSetDevice(prev);
}

// Lays out the class's global visited tables for `plan` (grow-only: a larger stride or more
// warps re-lays them out and zeroes them, so each warp keeps its table and epoch counter).
void Batcher::bind_visited(EfClass& c, const SearchPlan& plan) {
    if (plan.global_slots == 0) {
        return;
    }
    SearchArgs probe = args(c, SearchPlan{});
    const std::uint32_t warps = search_warps(probe, plan);
    if (c.d_visited == nullptr || plan.global_slots > c.visited_stride || warps > c.visited_warps) {
        const std::uint32_t stride = std::max(plan.global_slots, c.visited_stride);
        const std::uint32_t count = std::max(warps, c.visited_warps);
        const std::size_t bytes = global_visited_bytes(stride, count);
        if (c.d_visited != nullptr) {
            gpu::check(cudaDeviceSynchronize(), "visited tables");
            cudaFree(c.d_visited);
            c.d_visited = nullptr;
        }
        c.d_visited = gpu::device_alloc(bytes, "visited tables");
        gpu::check(cudaMemset(c.d_visited, 0, bytes), "clear visited tables");
        c.visited_stride = stride;
        c.visited_warps = count;
    }
}

SearchArgs Batcher::args(const EfClass& c, const SearchPlan& plan) {
    SearchArgs a;
    a.g = graph_view;
    a.queries = c.d_queries;
    a.nq = max_queries;   // capacity; the batch size is read from d_nq
    a.qstride = dim;
    a.nq_device = c.d_nq;
    a.k_per_q = c.d_k;
    a.ef_per_q = c.d_ef;
    a.k = max_k;
    a.ef = c.cap;
    a.out_stride = max_k;
    a.out_ids = c.d_ids;
    a.out_dists = c.d_dists;
    a.out_counts = c.d_counts;
    a.status = c.d_work;
    a.claim = c.d_work + 2;
    a.stats = reinterpret_cast<unsigned long long*>(c.d_work + 16);
    a.entry_ids = c.d_order;
    a.entry_d = reinterpret_cast<float*>(c.d_order + max_queries);
    a.order = c.d_order + 2 * static_cast<std::size_t>(max_queries);
    if (precision != Precision::FP32) {
        // As the batch search: an FP32 re-rank of the best 4 * k of each query.
        a.rerank = kRerankPerK * max_k;
        a.rerank_per_k = kRerankPerK;
    }
    if (plan.global_slots > 0 && c.d_visited != nullptr) {
        bind_global_visited(a, plan, c.d_visited, c.visited_stride, c.visited_warps);
    }
    return a;
}

void Batcher::enqueue(EfClass& c, const SearchPlan& p, cudaStream_t s) {
    gpu::check(cudaMemsetAsync(c.d_work, 0, kWorkWords * 4, s), "reset work words");
    gpu::check(cudaMemsetAsync(c.d_work + 1, 0xFF, 4, s), "reset work words");
    SearchArgs a = args(c, p);
    gpu::check(launch_search(a, p, s), "search kernel");
}

void Batcher::capture() {
    gpu::use_device(device);
    if (exec != nullptr) {
        cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
    if (graph != nullptr) {
        cudaGraphDestroy(graph);
        graph = nullptr;
    }
    for (EfClass& c : classes) {
        bind_visited(c, c.plan);  // allocation and clearing stay outside the capture
    }
    gpu::check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    gpu::check(cudaEventRecord(fork, stream), "fork");
    for (std::size_t i = 0; i < classes.size(); ++i) {
        gpu::check(cudaStreamWaitEvent(classes[i].stream, fork, 0), "fork");
        enqueue(classes[i], classes[i].plan, classes[i].stream);
        gpu::check(cudaEventRecord(joins[i], classes[i].stream), "join");
        gpu::check(cudaStreamWaitEvent(stream, joins[i], 0), "join");
    }
    gpu::check(cudaStreamEndCapture(stream, &graph), "end capture");
    gpu::check(cudaGraphInstantiate(&exec, graph, 0), "instantiate graph");
}

void Batcher::stage(const float* queries, std::uint32_t nq, const std::uint32_t* k,
                    const std::uint32_t* ef) {
    if (index.size() != index_size) {
        throw std::invalid_argument("Batcher: the index changed since the batcher was made");
    }
    if (nq > max_queries) {
        throw std::invalid_argument(std::format("Batcher: batch of {} exceeds the maximum {}", nq, max_queries));
    }
    for (EfClass& c : classes) {
        c.rows.clear();
    }
    const std::uint32_t n = classes.back().cap;  // min(max(max_ef, max_k), size)
    std::vector<std::uint32_t> eff(nq);
    for (std::uint32_t i = 0; i < nq; ++i) {
        if (k[i] == 0 || k[i] > max_k) {
            throw std::invalid_argument(std::format("Batcher: k {} outside [1, {}]", k[i], max_k));
        }
        std::uint64_t e = std::max(ef[i], k[i]);
        if (e > max_ef && e < index_size) {
            throw std::invalid_argument(std::format("Batcher: ef {} above the maximum {}", ef[i], max_ef));
        }
        // ef >= size searches exhaustively; every such query behaves alike.
        eff[i] = static_cast<std::uint32_t>(std::min<std::uint64_t>(e, std::min<std::uint64_t>(index_size, n)));
        std::size_t ci = 0;
        while (classes[ci].cap < eff[i]) {
            ++ci;
        }
        classes[ci].rows.push_back(i);
    }
    for (EfClass& c : classes) {
        std::stable_sort(c.rows.begin(), c.rows.end(),
                         [&](std::uint32_t x, std::uint32_t y) { return eff[x] > eff[y]; });
        const std::uint32_t m = static_cast<std::uint32_t>(c.rows.size());
        for (std::uint32_t j = 0; j < m; ++j) {
            const std::uint32_t i = c.rows[j];
            std::memcpy(c.h_queries + static_cast<std::size_t>(j) * dim,
                        queries + static_cast<std::size_t>(i) * dim, dim * 4ull);
            c.h_k[j] = k[i];
            c.h_ef[j] = ef[i];
        }
        *c.h_nq = m;
        if (m > 0) {
            gpu::check(cudaMemcpyAsync(c.d_queries, c.h_queries, static_cast<std::size_t>(m) * dim * 4,
                                       cudaMemcpyHostToDevice, stream), "copy queries");
            gpu::check(cudaMemcpyAsync(c.d_k, c.h_k, m * 4ull, cudaMemcpyHostToDevice, stream), "copy k");
            gpu::check(cudaMemcpyAsync(c.d_ef, c.h_ef, m * 4ull, cudaMemcpyHostToDevice, stream), "copy ef");
        }
        gpu::check(cudaMemcpyAsync(c.d_nq, c.h_nq, 4, cudaMemcpyHostToDevice, stream), "copy batch size");
    }
}

void Batcher::submit(const float* queries, std::uint32_t nq, const std::uint32_t* k,
                     const std::uint32_t* ef) {
    gpu::use_device(device);
    if (in_flight) {
        throw std::invalid_argument("Batcher::submit: the previous batch has not been collected (wait)");
    }
    stage(queries, nq, k, ef);
    gpu::check(cudaGraphLaunch(exec, stream), "graph launch");
    for (EfClass& c : classes) {
        const std::size_t m = c.rows.size();
        if (m > 0) {
            gpu::check(cudaMemcpyAsync(c.h_ids, c.d_ids, m * max_k * 4, cudaMemcpyDeviceToHost, stream),
                       "copy ids");
            gpu::check(cudaMemcpyAsync(c.h_dists, c.d_dists, m * max_k * 4, cudaMemcpyDeviceToHost, stream),
                       "copy distances");
            gpu::check(cudaMemcpyAsync(c.h_counts, c.d_counts, m * 4, cudaMemcpyDeviceToHost, stream),
                       "copy counts");
        }
        gpu::check(cudaMemcpyAsync(c.h_work, c.d_work, kWorkWords * 4, cudaMemcpyDeviceToHost, stream),
                   "copy status");
    }
    in_flight = true;
}

void Batcher::wait(std::uint32_t* ids, float* dists, std::uint32_t* counts) {
    gpu::use_device(device);
    if (!in_flight) {
        throw std::invalid_argument("Batcher::wait: no batch was submitted");
    }
    in_flight = false;
    gpu::check(cudaStreamSynchronize(stream), "batch");
    for (const EfClass& c : classes) {
        gpu::raise_status(c.h_work[0], "Batcher::run");
    }
    for (const EfClass& c : classes) {
        for (std::size_t j = 0; j < c.rows.size(); ++j) {
            const std::size_t i = c.rows[j];
            std::memcpy(ids + i * max_k, c.h_ids + j * max_k, max_k * 4ull);
            std::memcpy(dists + i * max_k, c.h_dists + j * max_k, max_k * 4ull);
            counts[i] = c.h_counts[j];
        }
    }
}

void Batcher::run(const float* queries, std::uint32_t nq, const std::uint32_t* k,
                  const std::uint32_t* ef, std::uint32_t* ids, float* dists,
                  std::uint32_t* counts) {
    submit(queries, nq, k, ef);
    wait(ids, dists, counts);
}

float Batcher::time_plan(EfClass& c, const SearchPlan& p, int reps) {
    bind_visited(c, p);
    cudaEvent_t a, b;
    gpu::check(cudaEventCreate(&a), "event");
    gpu::check(cudaEventCreate(&b), "event");
    enqueue(c, p, stream);  // warm-up
    gpu::check(cudaEventRecord(a, stream), "event");
    for (int i = 0; i < reps; ++i) {
        enqueue(c, p, stream);
    }
    gpu::check(cudaEventRecord(b, stream), "event");
    gpu::check(cudaEventSynchronize(b), "event");
    float ms = 0.0F;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    gpu::check(cudaMemcpy(c.h_work, c.d_work, kWorkWords * 4, cudaMemcpyDeviceToHost), "copy status");
    gpu::raise_status(c.h_work[0], "Batcher::autotune");
    return ms / static_cast<float>(reps);
}

std::vector<TunedPlan> Batcher::autotune(const float* queries, std::uint32_t nq,
                                         const std::uint32_t* k, const std::uint32_t* ef) {
    gpu::use_device(device);
    if (in_flight) {
        throw std::invalid_argument("Batcher::autotune: a batch is in flight (wait first)");
    }
    stage(queries, nq, k, ef);
    gpu::check(cudaStreamSynchronize(stream), "stage");
    std::vector<TunedPlan> tried;
    for (EfClass& c : classes) {
        if (c.rows.empty()) {
            continue;
        }
        // The visited-filter kind stays the default one (a global table from capacity 512): timed
        // alone, one batch is a little faster with the shared-memory table, but with batches in
        // flight on several batchers the global table's smaller per-warp footprint lets their
        // kernels share the SMs (2.3x the stream throughput on the uneven-stream workload).
        const std::vector<SearchPlan> bases{default_plan(graph_view, c.cap, true)};
        SearchPlan best = c.plan;
        float best_ms = -1.0F;
        for (const SearchPlan& base : bases) {
            const bool global = base.global_slots > 0;
            for (const int warps : {2, 4, 8}) {
                if (warps > max_warps_per_block(graph_view, base.efcap)) {
                    continue;
                }
                for (const std::uint32_t rows : {8u, 16u, 32u}) {
                    // Visited-filter size: shared-memory slots, or global slots for large ef.
                    const std::uint32_t mid = global ? base.global_slots : base.hash_slots;
                    for (const std::uint32_t slots : {mid / 2, mid, mid * 2}) {
                        if (slots < 512) {
                            continue;
                        }
                        SearchPlan p = base;
                        p.warps_per_block = warps;
                        p.rows_cap = std::max<std::uint32_t>(1, std::min(rows, graph_view.cap0));
                        (global ? p.global_slots : p.hash_slots) = slots;
                        SearchArgs a = args(c, p);
                        if (plan_search(a, p) > 200 * 1024) {
                            continue;
                        }
                        const float ms = time_plan(c, p, 3);
                        tried.push_back({c.cap, p, ms});
                        if (best_ms < 0.0F || ms < best_ms) {
                            best_ms = ms;
                            best = p;
                        }
                    }
                }
            }
        }
        c.plan = best;
    }
    capture();
    return tried;
}

}  // namespace vdx::dev
