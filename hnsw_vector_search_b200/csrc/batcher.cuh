#pragma once

// Uneven batches through one captured CUDA graph, with an autotuned launch plan per ef class
// (batcher.cu).

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "search.cuh"
#include "vdx/hnsw.hpp"

namespace vdx::dev {

struct TunedPlan {
    std::uint32_t ef_class;   // the class's result-list capacity
    SearchPlan plan;
    float ms;
};

// One ef class: queries whose effective ef is at most `cap`, with their own launch plan and
// fixed device / pinned buffers for up to max_queries rows.
struct EfClass {
    std::uint32_t cap = 0;
    SearchPlan plan{};
    cudaStream_t stream = nullptr;        // capture branch
    float* d_queries = nullptr;
    std::uint32_t *d_k = nullptr, *d_ef = nullptr, *d_nq = nullptr, *d_ids = nullptr,
                  *d_counts = nullptr, *d_work = nullptr;
    float* d_dists = nullptr;
    float* h_queries = nullptr;
    std::uint32_t *h_k = nullptr, *h_ef = nullptr, *h_nq = nullptr, *h_ids = nullptr,
                  *h_counts = nullptr, *h_work = nullptr;
    float* h_dists = nullptr;
    std::vector<std::uint32_t> rows;      // batch row of each staged position
    std::uint32_t* d_order = nullptr;     // ordered-launch scratch: 3 words per query
    void* d_visited = nullptr;            // global visited tables (large-ef plans), grow-only
    std::uint32_t visited_stride = 0;
    std::uint32_t visited_warps = 0;
};

struct Batcher {
    Batcher(const HnswIndex& index, int device, Precision precision, std::uint32_t max_queries,
            std::uint32_t max_k, std::uint32_t max_ef);
    ~Batcher();
    Batcher(const Batcher&) = delete;
    Batcher& operator=(const Batcher&) = delete;

    // One batch (host buffers): queries nq x dim, per-query k and ef; results nq x max_k.
    void run(const float* queries, std::uint32_t nq, const std::uint32_t* k, const std::uint32_t* ef,
             std::uint32_t* ids, float* dists, std::uint32_t* counts);
    // The same in two halves: submit stages the batch and enqueues the copies and the graph on
    // this batcher's stream without waiting (the caller's buffers may be reused at once); wait
    // blocks until that batch is done and writes its results. One batch in flight per batcher;
    // several batchers keep several batches in flight.
    void submit(const float* queries, std::uint32_t nq, const std::uint32_t* k, const std::uint32_t* ef);
    void wait(std::uint32_t* ids, float* dists, std::uint32_t* counts);
    bool in_flight = false;
    // Times the candidate plans of every class on this batch, keeps each class's fastest and
    // re-captures the graph.
    std::vector<TunedPlan> autotune(const float* queries, std::uint32_t nq, const std::uint32_t* k,
                                    const std::uint32_t* ef);

    const HnswIndex& index;
    int device;
    Precision precision;
    std::uint32_t max_queries, max_k, max_ef, dim = 0;
    std::size_t index_size = 0;
    DeviceGraphView graph_view{};
    std::vector<EfClass> classes;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

private:
    SearchArgs args(const EfClass& c, const SearchPlan& plan);
    void bind_visited(EfClass& c, const SearchPlan& plan);
    void enqueue(EfClass& c, const SearchPlan& plan, cudaStream_t stream);
    void capture();
    void stage(const float* queries, std::uint32_t nq, const std::uint32_t* k, const std::uint32_t* ef);
    float time_plan(EfClass& c, const SearchPlan& plan, int reps);
};

}  // namespace vdx::dev
