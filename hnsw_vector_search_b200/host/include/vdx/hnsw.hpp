#pragma once

// The HNSW index. Its public API is the reference's (include/vecdex/hnsw.hpp:63-123: constructor,
// add, search, search_batch, inspect, memory_bytes, save, load) so that a caller switches by
// changing the namespace; the graph it holds, and the file it saves, are the reference's too
// (docs/FORMAT.md v1), so an index saved by the reference loads here unchanged and the other way
// round.
//
// What differs is where queries run. search() and search_batch() run on a B200: a device mirror
// of the graph (vdx/device.hpp) is uploaded on first use and refreshed after add(), and every
// query distance, traversal step and result merge runs in hand-written sm_100a kernels. There is
// no CPU search path. Graph construction (add) runs on the host, as in the reference, and is the
// only place host code computes distances.

#include <cstddef>
#include <cstdint>
#include <filesystem>
#include <memory>
#include <mutex>
#include <random>
#include <span>
#include <string>
#include <vector>

#include "vdx/distance.hpp"
#include "vdx/matrix.hpp"
#include "vdx/neighbor.hpp"

namespace vdx {

struct DeviceGraph;  // vdx/device.hpp
namespace dev {
struct DeviceStopNet;
}

// The learned early-termination model (12 -> 64 -> 64 -> 1): 5,057 FP32 parameters, the
// feature standardization, and the 4 random projection directions (4 rows of dim floats).
struct StopModel {
    std::vector<float> weights;
    std::vector<float> mean;
    std::vector<float> inv_std;
    std::vector<float> proj;
};

struct HnswParams {
    std::size_t M = 16;                            // links per node per layer; 2M on layer 0
    static constexpr std::size_t kMaxM = 10'000;   // the reference's limit
    std::size_t ef_construction = 200;             // candidate list size while inserting
    std::uint64_t seed = 42;                       // seeds the level generator
};

struct GraphReport {
    std::vector<std::string> violations;
    std::size_t reachable = 0;  // layer-0 nodes reachable from the entry point
    std::size_t max_level = 0;
    double mean_degree0 = 0.0;
};

// Element type of the vector copy the layer-0 traversal reads (SearchOptions::precision).
enum class Precision : std::uint8_t {
    FP32 = 0,  // the stored vectors: distances bit-identical to the reference's
    BF16 = 1,  // bfloat16 copy, FP32 accumulation; results re-ranked in FP32
    FP8 = 2,   // FP8 E4M3 copy with one FP32 scale per vector; re-ranked in FP32
};

// GPU search knobs beyond the reference API. The defaults give the reference's results.
struct SearchOptions {
    Precision precision = Precision::FP32;
    // For BF16 / FP8: how many of the best candidates are re-scored in FP32 before the top k is
    // taken; 0 means 4k, kNoRerank none (the traversal-precision distances are returned).
    std::uint32_t rerank = 0;
    // Learned early termination: a small network, evaluated in the kernel every 8 expansions,
    // stops a query's layer-0 search once it predicts the top k has converged. Needs a model
    // (HnswIndex::set_stop_model); ef stays the hard cap.
    bool learned_stop = false;
    float stop_threshold = 0.5F;
    // Consult the network only once the k-th distance has been unchanged for this many
    // expansions in a row (0 to 3; 0: at every checkpoint).
    std::uint32_t stop_gate = 0;
    int device = 0;
};

inline constexpr std::uint32_t kNoRerank = 0xFFFFFFFFu;

// The FP32 re-rank width a search with `options` and k uses (0: none).
inline std::uint32_t rerank_width(const SearchOptions& options, std::size_t k) {
    if (options.precision == Precision::FP32 || options.rerank == kNoRerank) {
        return 0;
    }
    return options.rerank > 0 ? options.rerank : static_cast<std::uint32_t>(4 * k);
}

class HnswIndex {
public:
    explicit HnswIndex(std::size_t dim, Metric metric = Metric::L2, HnswParams params = {});
    ~HnswIndex();
    HnswIndex(HnswIndex&&) noexcept;
    HnswIndex& operator=(HnswIndex&&) noexcept;
    HnswIndex(const HnswIndex&) = delete;
    HnswIndex& operator=(const HnswIndex&) = delete;

    std::size_t dim() const noexcept { return vectors_.dim(); }
    std::size_t size() const noexcept { return vectors_.rows(); }
    Metric metric() const noexcept { return metric_; }
    const HnswParams& params() const noexcept { return params_; }

    // Graph construction on the host, the reference's algorithm (serial builds are identical to
    // the reference's, byte for byte once saved).
    Id add(std::span<const float> vector);
    void add(MatrixView<float> vectors, std::size_t num_threads = 1);
    // The same insertion, batched on the GPU (device `device`): the first 1024 nodes one by one
    // on the host as the serial build, then batches of up to 8192 nodes searched, linked and
    // linked back by kernels, with the serial order's levels. The graph is as good as a parallel
    // build's (recall within 0.005 of the serial build), not the serial graph itself; the FP32
    // device mirror is built in place.
    void add_gpu(MatrixView<float> vectors, int device);
    void add(const Matrix<float>& vectors, std::size_t num_threads = 1);

    // Up to k nearest neighbors, closest first, ties by smaller id; ef below k is raised to k.
    // Runs on the GPU.
    std::vector<Neighbor> search(std::span<const float> query, std::size_t k, std::size_t ef) const;

    // search() for every row, as one GPU batch. Element i equals search(row i). num_threads is
    // accepted for source compatibility and ignored: the batch is one launch.
    std::vector<std::vector<Neighbor>> search_batch(MatrixView<float> queries, std::size_t k,
                                                    std::size_t ef,
                                                    std::size_t num_threads = 0) const;

    // search_batch into caller buffers of queries.rows() * k entries (ids, distances) and
    // queries.rows() counts; rows shorter than k are padded with id 0xFFFFFFFF and +inf.
    // `where` names the calling API in error messages.
    void search_batch_into(MatrixView<float> queries, std::size_t k, std::size_t ef, Id* ids,
                           float* distances, std::uint32_t* counts,
                           const SearchOptions& options = {},
                           const char* where = "HnswIndex::search_batch") const;

    GraphReport inspect() const;
    std::size_t memory_bytes() const noexcept;

    void save(const std::filesystem::path& path) const;
    static HnswIndex load(const std::filesystem::path& path);

    // The device mirror for `device`, uploaded (or refreshed after add()) on first use.
    // Thread-safe; the returned reference stays valid until the next add() or destruction.
    const DeviceGraph& device_graph(int device, Precision precision) const;
    // The device mirror for `device` if it is already uploaded and current, else nullptr.
    // Never uploads, so it never allocates.
    const DeviceGraph* uploaded_graph(int device, Precision precision) const;

    // The FP32 device mirror as a sidecar file beside the v1 index file: the device arrays in
    // their device layout, each section 4096-byte aligned, behind a 4096-byte header that names
    // the graph by graph_hash(). save_device_image() runs on the host only;
    // load_device_image() installs the file as the FP32 mirror for `device` with one copy per
    // section (no repacking), and throws std::runtime_error if the file belongs to another
    // graph, is truncated or is not a device image.
    void save_device_image(const std::filesystem::path& path) const;
    void load_device_image(const std::filesystem::path& path, int device) const;
    // XXH64 of the vectors, levels, layer-0 blocks and upper blocks, in that order.
    std::uint64_t graph_hash() const;

    // Learned early termination: the model SearchOptions::learned_stop uses.
    void set_stop_model(StopModel model);
    bool has_stop_model() const noexcept { return !stop_model_.weights.empty(); }
    const StopModel& stop_model() const noexcept { return stop_model_; }
    // The model's device copy for `device`, uploaded on first use (throws without a model).
    const dev::DeviceStopNet& stop_net(int device) const;

    // Training traces: the plain search of every query at `ef`; every 8 expansions the 12
    // features of its state (projections from `proj`, 4 rows of dim floats) and how many of its
    // current top k are in `truth` (truth_k ids per query), and at the end the final hits.
    // Buffers: features [nq][max_points][12], hits [nq][max_points], points [nq], final [nq].
    void trace_search(MatrixView<float> queries, const Id* truth, std::size_t truth_k,
                      std::size_t k, std::size_t ef, const float* proj, std::size_t max_points,
                      float* features, std::uint8_t* hits, std::uint32_t* points,
                      std::uint8_t* final_hits, int device = 0) const;

    // Read-only views of the graph, in the reference's in-memory layout.
    std::span<const std::uint8_t> levels() const noexcept { return levels_; }
    std::span<const Id> layer0() const noexcept { return layer0_; }
    std::span<const Id> upper_blocks(Id node) const noexcept { return upper_[node]; }
    std::span<const float> vectors() const noexcept { return vectors_.data(); }
    Id entry_point() const noexcept { return entry_point_; }
    std::size_t max_level() const noexcept { return max_level_; }

private:
    struct ListGuards;  // mutexes of a parallel add (hnsw_build.cpp)
    class Builder;      // the insertion procedure (hnsw_build.cpp)

    std::size_t max_links(std::size_t layer) const noexcept {
        return layer == 0 ? 2 * params_.M : params_.M;
    }
    // A node's link block on `layer`: [count, ids...], 1 + max_links(layer) words.
    std::span<Id> block(Id node, std::size_t layer) noexcept;
    std::span<const Id> block(Id node, std::size_t layer) const noexcept;
    // The links of a block (its first `count` ids); the count must be within capacity.
    std::span<const Id> links(Id node, std::size_t layer) const noexcept;
    float dist(const float* a, const float* b) const noexcept;
    const float* vector_of(Id node) const noexcept { return vectors_.row(node).data(); }

    std::size_t draw_level();
    // Stores a vector (normalized under cosine), draws its level and lays out empty link blocks.
    void append_node(std::span<const float> vector);
    // Inserts a stored node into the graph on the calling thread (the serial build's step).
    void link_serial(Id node);
    void check_links(const std::filesystem::path& path) const;
    void invalidate_device() noexcept;

    Metric metric_;
    HnswParams params_;
    double level_multiplier_;
    std::mt19937_64 rng_;
    Matrix<float> vectors_;  // unit length under Cosine
    std::vector<std::uint8_t> levels_;
    std::vector<Id> layer0_;              // n blocks of [count, ids... (2M)]
    std::vector<std::vector<Id>> upper_;  // per node: blocks of [count, ids... (M)], layers 1..level
    Id entry_point_ = 0;
    std::size_t max_level_ = 0;

    ListGuards* guards_ = nullptr;  // set only while a parallel add runs
    mutable std::unique_ptr<std::mutex> device_mutex_;
    mutable std::vector<std::unique_ptr<DeviceGraph>> device_;  // per (device, precision) slot
    StopModel stop_model_;
    mutable std::vector<std::shared_ptr<dev::DeviceStopNet>> stop_net_;  // per device
};

}  // namespace vdx
