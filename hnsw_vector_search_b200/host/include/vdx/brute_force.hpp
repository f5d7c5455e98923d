#pragma once

// Exact k-nearest-neighbor search, the reference's BruteForceIndex
// (include/vecdex/brute_force.hpp:21-43) with the same API and results; search runs on the GPU
// (vectors are uploaded on first use and after add()).

#include <cstddef>
#include <cstdint>
#include <memory>
#include <mutex>
#include <span>
#include <vector>

#include "vdx/distance.hpp"
#include "vdx/matrix.hpp"
#include "vdx/neighbor.hpp"

namespace vdx {

struct DeviceBase;

// Which kernel scores the batch.
enum class BruteMethod : std::uint8_t {
    Exact = 0,        // CUDA cores, every distance in the reference's FP32 order
    TensorCore = 1,   // tcgen05 split-BF16 GEMM candidates, exact re-rank, certified: the same
                      // ids and distance bits as Exact (shapes it does not cover run Exact); the
                      // default
};

class BruteForceIndex {
public:
    explicit BruteForceIndex(std::size_t dim, Metric metric = Metric::L2);
    ~BruteForceIndex();
    BruteForceIndex(BruteForceIndex&&) noexcept;
    BruteForceIndex& operator=(BruteForceIndex&&) noexcept;

    std::size_t dim() const noexcept { return vectors_.dim(); }
    std::size_t size() const noexcept { return vectors_.rows(); }
    Metric metric() const noexcept { return metric_; }

    Id add(std::span<const float> vector);
    void add(const Matrix<float>& vectors);
    void add(MatrixView<float> vectors);

    // The min(k, size()) closest stored vectors, closest first, ties by smaller id.
    std::vector<Neighbor> search(std::span<const float> query, std::size_t k) const;

    // search() for every row, one GPU batch, into caller buffers (padded like
    // HnswIndex::search_batch_into).
    void search_batch_into(MatrixView<float> queries, std::size_t k, Id* ids, float* distances,
                           std::uint32_t* counts, BruteMethod method = BruteMethod::TensorCore,
                           int device = 0, const char* where = "BruteForceIndex::search") const;

    // The device-buffer form: queries, results and the work words (status, first failing row,
    // uncertified count at word 8) in device memory, asynchronous on `stream`.
    void search_batch_device(const float* d_queries, std::size_t nq, std::size_t dim,
                             std::size_t k, Id* d_ids, float* d_dists, std::uint32_t* d_counts,
                             std::uint32_t* d_work, BruteMethod method, void* stream,
                             int device = 0) const;

    std::span<const float> vectors() const noexcept { return vectors_.data(); }
    const DeviceBase& device_base(int device) const;

private:
    void store(std::span<const float> values);

    Metric metric_;
    Matrix<float> vectors_;
    mutable std::unique_ptr<std::mutex> device_mutex_;
    mutable std::vector<std::unique_ptr<DeviceBase>> device_;
};

}  // namespace vdx
