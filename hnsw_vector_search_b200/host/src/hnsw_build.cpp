// HnswIndex construction and diagnostics on the host.
//
// The graph has to be the one the reference builds, so that a serial build here saves the same
// file byte for byte and GPU results can be compared id for id with the reference's on either
// build. What fixes the graph is the algorithm, which follows the HNSW paper (Malkov & Yashunin,
// 2018) with the reference's choices (src/hnsw.cpp:223-409):
//   * level of a new node: floor(-ln U * 1/ln M), U = 1 - (top 53 bits of the next mt19937_64
//     output) * 2^-53, drawn when the vector is stored (paper Alg. 1, line 4);
//   * insertion (Alg. 1): from the entry point, a greedy walk through the layers above the node's
//     level, moving to the first strict minimum of each scanned neighbour list (distance only)
//     until no move is made; then, on every layer from min(level, top) down to 0, a best-first
//     search with ef = max(ef_construction, M) (Alg. 2) whose closest result seeds the next
//     layer, and M neighbours selected from its results by the heuristic of Alg. 4 (no
//     extension, no pruned-connection refill);
//   * neighbour lists of the chosen nodes: the new node is appended while a list has room,
//     otherwise the list is re-selected by the same heuristic from its old links plus the new
//     node, at its capacity (2M on layer 0, M above);
//   * order: (distance, id) as Neighbor's `closer` defines it, everywhere.
//
// How the code gets there is this project's own. The layer search keeps one sorted beam with an
// "expanded" mark per entry instead of a candidate heap and a result heap: expanding the closest
// unexpanded beam entry until none is left visits the same nodes in the same order and ends with
// the same results (a candidate evicted from the results would only ever stop the heap search,
// at the point where the beam has nothing left to expand). It is the same loop the GPU search
// kernel runs. A parallel add stores every vector first (levels in the serial order), then
// inserts the rest from worker threads that claim chunks of nodes; neighbour lists are guarded
// by a fixed table of striped mutexes, at most one held at a time, and a node that raises the
// top layer holds the entry-point mutex through its whole insertion.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <exception>
#include <format>
#include <mutex>
#include <optional>
#include <stdexcept>
#include <thread>
#include <utility>

#include "internal.hpp"
#include "vdx/device.hpp"
#include "vdx/hnsw.hpp"

namespace vdx {

// Mutexes of a parallel add: neighbour lists hash to one of a fixed number of stripes.
struct HnswIndex::ListGuards {
    static constexpr std::size_t kStripes = std::size_t{1} << 14;
    std::mutex stripe[kStripes];
    std::mutex top;  // entry point and top layer
    std::mutex& of(Id node) noexcept { return stripe[(node * 0x9E3779B1u) >> 18]; }
};

// One inserting thread's procedure and scratch.
class HnswIndex::Builder {
public:
    Builder(HnswIndex& index, ListGuards* guards) : ix_(index), guards_(guards) {}

    void insert(Id node);
    const HnswIndex& index() const noexcept { return ix_; }
    const ListGuards* guards() const noexcept { return guards_; }

private:
    struct Entry {
        Neighbor n;
        bool expanded;
    };

    std::span<const Id> neighbours(Id node, std::size_t layer);
    Neighbor walk(const float* q, Neighbor at, std::size_t layer);
    void layer_search(const float* q, Neighbor from, std::size_t ef, std::size_t layer);
    std::vector<Neighbor> diverse(std::span<const Neighbor> sorted, std::size_t m) const;
    void link_from(Id node, std::size_t layer, const Neighbor& to);
    bool first_visit(Id id);

    HnswIndex& ix_;
    ListGuards* guards_;
    std::vector<Id> list_copy_;
    std::vector<std::uint32_t> mark_;
    std::uint32_t epoch_ = 0;
    std::vector<Entry> beam_;
    std::vector<Neighbor> sorted_;
};

namespace {

HnswParams validated(const HnswParams& p) {
    if (p.M < 2) {
        throw std::invalid_argument("HnswIndex: M must be at least 2");
    }
    if (p.M > HnswParams::kMaxM) {
        throw std::invalid_argument(
            std::format("HnswIndex: M must be at most {}", HnswParams::kMaxM));
    }
    if (p.ef_construction == 0) {
        throw std::invalid_argument("HnswIndex: ef_construction must be positive");
    }
    return p;
}

// Runs body(begin, end) over [0, count) on up to `threads` threads, each claiming chunks of 64
// items; after every thread has stopped, the first error (in thread order) is rethrown.
template <typename Body>
void for_chunks(std::size_t count, std::size_t threads, const Body& body) {
    constexpr std::size_t kChunk = 64;
    std::atomic<std::size_t> cursor{0};
    std::atomic<bool> failed{false};
    const std::size_t workers = std::max<std::size_t>(1, std::min(threads, (count + kChunk - 1) / kChunk));
    std::vector<std::optional<std::exception_ptr>> errors(workers);
    const auto run = [&](std::size_t w) {
        try {
            while (!failed.load(std::memory_order_relaxed)) {
                const std::size_t begin = cursor.fetch_add(kChunk);
                if (begin >= count) {
                    return;
                }
                body(begin, std::min(count, begin + kChunk));
            }
        } catch (...) {
            errors[w] = std::current_exception();
            failed = true;
        }
    };
    {
        std::vector<std::jthread> pool;
        pool.reserve(workers - 1);
        for (std::size_t w = 1; w < workers; ++w) {
            pool.emplace_back(run, w);
        }
        run(0);
    }  // joins
    for (const auto& e : errors) {
        if (e) {
            std::rethrow_exception(*e);
        }
    }
}

}  // namespace

HnswIndex::HnswIndex(std::size_t dim, Metric metric, HnswParams params)
    : metric_(metric), params_(validated(params)), vectors_(dim) {
    level_multiplier_ = 1.0 / std::log(static_cast<double>(params_.M));
    rng_.seed(params_.seed);
    device_mutex_ = std::make_unique<std::mutex>();
}

HnswIndex::~HnswIndex() = default;
HnswIndex::HnswIndex(HnswIndex&&) noexcept = default;
HnswIndex& HnswIndex::operator=(HnswIndex&&) noexcept = default;

// Storage: layer 0 is one array of n blocks, every node's upper layers one vector of `level`
// blocks; a block is [count, ids...] with room for max_links(layer) ids.
std::span<const Id> HnswIndex::block(Id node, std::size_t layer) const noexcept {
    const std::size_t width = 1 + max_links(layer);
    const Id* base = layer == 0 ? layer0_.data() + static_cast<std::size_t>(node) * width
                                : upper_[node].data() + (layer - 1) * width;
    return {base, width};
}

std::span<Id> HnswIndex::block(Id node, std::size_t layer) noexcept {
    const std::span<const Id> b = std::as_const(*this).block(node, layer);
    return {const_cast<Id*>(b.data()), b.size()};
}

std::span<const Id> HnswIndex::links(Id node, std::size_t layer) const noexcept {
    const std::span<const Id> b = block(node, layer);
    return b.subspan(1, b[0]);
}

float HnswIndex::dist(const float* a, const float* b) const noexcept {
    return metric_ == Metric::L2 ? detail::l2_squared_raw(a, b, dim())
                                 : 1.0F - detail::inner_product_raw(a, b, dim());
}

std::size_t HnswIndex::memory_bytes() const noexcept {
    // Every node's upper vector holds exactly level x (1 + M) ids (append_node() and load() size
    // them so), which lets the levels give the total without visiting n separate allocations.
    std::size_t upper_blocks = 0;
    for (const std::uint8_t level : levels_) {
        upper_blocks += level;
    }
    return vectors_.data().size_bytes() + levels_.size() + layer0_.size() * sizeof(Id) +
           upper_.size() * sizeof(std::vector<Id>) +
           upper_blocks * (1 + max_links(1)) * sizeof(Id);
}

void HnswIndex::invalidate_device() noexcept {
    if (device_mutex_) {
        const std::scoped_lock lock(*device_mutex_);
        device_.clear();
    }
}

std::size_t HnswIndex::draw_level() {
    const std::uint64_t top53 = rng_() >> 11U;
    const double u = 1.0 - std::ldexp(static_cast<double>(top53), -53);  // in (0, 1]
    return static_cast<std::size_t>(-std::log(u) * level_multiplier_);
}

void HnswIndex::append_node(std::span<const float> vector) {
    if (device_mutex_ == nullptr) {  // a moved-from index being reused
        device_mutex_ = std::make_unique<std::mutex>();
    }
    const std::size_t id = size();
    vectors_.append(vector);
    if (metric_ == Metric::Cosine) {
        detail::normalize(vectors_.row(id));
    }
    const std::size_t level = draw_level();
    levels_.push_back(static_cast<std::uint8_t>(level));
    layer0_.insert(layer0_.end(), 1 + max_links(0), Id{0});
    upper_.push_back(std::vector<Id>(level * (1 + max_links(1)), Id{0}));
}

void HnswIndex::link_serial(Id node) {
    thread_local std::unique_ptr<Builder> builder;
    if (builder == nullptr || &builder->index() != this) {
        builder = std::make_unique<Builder>(*this, nullptr);
    }
    builder->insert(node);
}

Id HnswIndex::add(std::span<const float> vector) {
    detail::check_new_vectors("HnswIndex::add", {metric_, dim(), size()}, vector.size(), vector);
    invalidate_device();
    append_node(vector);
    const auto id = static_cast<Id>(size() - 1);
    link_serial(id);
    return id;
}

void HnswIndex::add(const Matrix<float>& vectors, std::size_t num_threads) {
    add(MatrixView<float>(vectors), num_threads);
}

void HnswIndex::add(MatrixView<float> vectors, std::size_t num_threads) {
    detail::check_new_vectors("HnswIndex::add", {metric_, dim(), size()}, vectors.dim(),
                              vectors.data());
    invalidate_device();
    const std::size_t rows = vectors.rows();
    const std::size_t first = size();
    vectors_.reserve_rows(first + rows);
    levels_.reserve(first + rows);
    layer0_.reserve((first + rows) * (1 + max_links(0)));
    upper_.reserve(first + rows);
    const std::size_t threads =
        num_threads == 0 ? std::max(1U, std::thread::hardware_concurrency()) : num_threads;
    if (threads == 1 || rows <= 1) {
        for (std::size_t r = 0; r < rows; ++r) {
            append_node(vectors.row(r));
            link_serial(static_cast<Id>(first + r));
        }
        return;
    }
    // All vectors stored (and levels drawn in the serial order) before any link is made, so no
    // container is resized while workers read it.
    for (std::size_t r = 0; r < rows; ++r) {
        append_node(vectors.row(r));
    }
    std::size_t start = first;
    if (start == 0) {
        link_serial(0);  // the first node only becomes the entry point
        start = 1;
    }
    auto guards = std::make_unique<ListGuards>();
    guards_ = guards.get();
    try {
        for_chunks(size() - start, threads, [&](std::size_t begin, std::size_t end) {
            thread_local std::unique_ptr<Builder> builder;
            if (builder == nullptr || &builder->index() != this || builder->guards() != guards_) {
                builder = std::make_unique<Builder>(*this, guards_);
            }
            for (std::size_t i = begin; i < end; ++i) {
                builder->insert(static_cast<Id>(start + i));
            }
        });
    } catch (...) {
        guards_ = nullptr;
        throw;
    }
    guards_ = nullptr;
}

// ---------------------------------------------------------------------------------------------
// The insertion procedure.

bool HnswIndex::Builder::first_visit(Id id) {
    if (mark_[id] == epoch_) {
        return false;
    }
    mark_[id] = epoch_;
    return true;
}

// A node's neighbour list on `layer`; under a parallel add a copy taken under its stripe.
std::span<const Id> HnswIndex::Builder::neighbours(Id node, std::size_t layer) {
    if (guards_ == nullptr) {
        return ix_.links(node, layer);
    }
    const std::scoped_lock lock(guards_->of(node));
    const std::span<const Id> now = ix_.links(node, layer);
    list_copy_.assign(now.begin(), now.end());
    return list_copy_;
}

// Greedy walk on one layer: score the whole list of the current node, move to its first strict
// minimum if that beats the current distance, repeat until no move.
Neighbor HnswIndex::Builder::walk(const float* q, Neighbor at, std::size_t layer) {
    for (;;) {
        Neighbor best = at;
        for (const Id id : neighbours(at.id, layer)) {
            const float d = ix_.dist(q, ix_.vector_of(id));
            if (d < best.distance) {
                best = {d, id};
            }
        }
        if (best.id == at.id) {
            return at;
        }
        at = best;
    }
}

// Best-first search of one layer into beam_: at most ef entries, sorted by `closer`.
void HnswIndex::Builder::layer_search(const float* q, Neighbor from, std::size_t ef,
                                      std::size_t layer) {
    if (mark_.size() < ix_.size()) {
        mark_.resize(ix_.size(), 0);
    }
    if (++epoch_ == 0) {
        std::ranges::fill(mark_, 0U);
        epoch_ = 1;
    }
    first_visit(from.id);
    beam_.assign(1, Entry{from, false});
    std::size_t cursor = 0;  // no unexpanded entry before this position
    for (;;) {
        while (cursor < beam_.size() && beam_[cursor].expanded) {
            ++cursor;
        }
        if (cursor == beam_.size()) {
            return;
        }
        beam_[cursor].expanded = true;
        const Id node = beam_[cursor].n.id;
        for (const Id id : neighbours(node, layer)) {
            if (!first_visit(id)) {
                continue;
            }
            const Neighbor cand{ix_.dist(q, ix_.vector_of(id)), id};
            const bool full = beam_.size() >= ef;
            if (full && !closer(cand, beam_.back().n)) {
                continue;
            }
            const auto at = std::ranges::upper_bound(beam_, cand, closer, &Entry::n);
            const auto pos = static_cast<std::size_t>(at - beam_.begin());
            beam_.insert(at, Entry{cand, false});
            if (full) {
                beam_.pop_back();
            }
            cursor = std::min(cursor, pos);
        }
    }
}

// Paper Alg. 4 over candidates sorted by `closer`: a candidate is kept unless some kept node is
// closer to it than the base node is; at most m kept; m or fewer candidates are all kept.
std::vector<Neighbor> HnswIndex::Builder::diverse(std::span<const Neighbor> sorted,
                                                  std::size_t m) const {
    if (sorted.size() <= m) {
        return {sorted.begin(), sorted.end()};
    }
    std::vector<Neighbor> kept;
    kept.reserve(m);
    for (std::size_t i = 0; i < sorted.size() && kept.size() < m; ++i) {
        const float* v = ix_.vector_of(sorted[i].id);
        const bool dominated = std::ranges::any_of(kept, [&](const Neighbor& k) {
            return ix_.dist(v, ix_.vector_of(k.id)) < sorted[i].distance;
        });
        if (!dominated) {
            kept.push_back(sorted[i]);
        }
    }
    return kept;
}

// Adds `node` (at distance to.distance) to the list of `to.id` on `layer`: appended while the
// list has room, else the list is re-selected from its links plus `node`.
void HnswIndex::Builder::link_from(Id node, std::size_t layer, const Neighbor& to) {
    std::unique_lock<std::mutex> lock;
    if (guards_ != nullptr) {
        lock = std::unique_lock(guards_->of(to.id));
    }
    const std::span<Id> b = ix_.block(to.id, layer);
    const std::size_t cap = ix_.max_links(layer);
    if (b[0] < cap) {
        b[1 + b[0]] = node;
        ++b[0];
        return;
    }
    const float* owner = ix_.vector_of(to.id);
    sorted_.clear();
    for (std::size_t i = 1; i <= b[0]; ++i) {
        sorted_.push_back({ix_.dist(owner, ix_.vector_of(b[i])), b[i]});
    }
    sorted_.push_back({to.distance, node});
    std::ranges::sort(sorted_, closer);
    const std::vector<Neighbor> kept = diverse(sorted_, cap);
    b[0] = static_cast<Id>(kept.size());
    std::ranges::transform(kept, b.begin() + 1, &Neighbor::id);
}

void HnswIndex::Builder::insert(Id node) {
    const std::size_t level = ix_.levels_[node];
    if (node == 0) {
        ix_.entry_point_ = 0;
        ix_.max_level_ = level;
        return;
    }
    std::unique_lock<std::mutex> top;
    if (guards_ != nullptr) {
        top = std::unique_lock(guards_->top);
    }
    const Id entry = ix_.entry_point_;
    const std::size_t top_level = ix_.max_level_;
    const bool raises_top = level > top_level;
    if (top.owns_lock() && !raises_top) {
        top.unlock();
    }
    const float* q = ix_.vector_of(node);
    Neighbor at{ix_.dist(q, ix_.vector_of(entry)), entry};
    for (std::size_t layer = top_level; layer > level; --layer) {
        at = walk(q, at, layer);
    }
    const std::size_t ef = std::max(ix_.params_.ef_construction, ix_.params_.M);
    const std::size_t highest = std::min(level, top_level);
    std::vector<std::vector<Neighbor>> chosen(highest + 1);
    for (std::size_t layer = highest + 1; layer-- > 0;) {
        layer_search(q, at, ef, layer);
        at = beam_.front().n;
        sorted_.clear();
        std::ranges::transform(beam_, std::back_inserter(sorted_), &Entry::n);
        chosen[layer] = diverse(sorted_, ix_.params_.M);
    }
    {
        std::unique_lock<std::mutex> own;
        if (guards_ != nullptr) {
            own = std::unique_lock(guards_->of(node));
        }
        for (std::size_t layer = 0; layer <= highest; ++layer) {
            const std::span<Id> b = ix_.block(node, layer);
            b[0] = static_cast<Id>(chosen[layer].size());
            std::ranges::transform(chosen[layer], b.begin() + 1, &Neighbor::id);
        }
    }
    for (std::size_t layer = 0; layer <= highest; ++layer) {
        for (const Neighbor& to : chosen[layer]) {
            link_from(node, layer, to);
        }
    }
    if (raises_top) {
        ix_.max_level_ = level;
        ix_.entry_point_ = node;
    }
}

// ---------------------------------------------------------------------------------------------

GraphReport HnswIndex::inspect() const {
    GraphReport r;
    r.max_level = max_level_;
    const std::size_t n = size();
    if (n == 0) {
        return r;
    }
    std::size_t highest = 0;
    std::size_t degree0 = 0;
    std::vector<Id> sorted;
    for (Id node = 0; node < n; ++node) {
        const std::size_t level = levels_[node];
        highest = std::max(highest, level);
        for (std::size_t layer = 0; layer <= level; ++layer) {
            const auto ids = links(node, layer);
            if (layer == 0) {
                degree0 += ids.size();
            }
            if (ids.size() > max_links(layer)) {
                r.violations.push_back(std::format("node {} has {} links on layer {} (max {})",
                                                   node, ids.size(), layer, max_links(layer)));
            }
            sorted.assign(ids.begin(), ids.end());
            std::ranges::sort(sorted);
            if (std::ranges::adjacent_find(sorted) != sorted.end()) {
                r.violations.push_back(
                    std::format("node {} has a duplicate link on layer {}", node, layer));
            }
            for (const Id id : ids) {
                if (id == node) {
                    r.violations.push_back(
                        std::format("node {} links to itself on layer {}", node, layer));
                } else if (id >= n) {
                    r.violations.push_back(std::format("node {} links to missing node {}", node, id));
                } else if (levels_[id] < layer) {
                    r.violations.push_back(std::format(
                        "node {} links to node {} on layer {}, above its level", node, id, layer));
                }
            }
        }
    }
    if (highest != max_level_) {
        r.violations.push_back(
            std::format("max level is {} but the tallest node reaches {}", max_level_, highest));
    }
    if (levels_[entry_point_] != max_level_) {
        r.violations.push_back(
            std::format("entry point {} is not on the top layer", entry_point_));
    }
    std::vector<bool> seen(n, false);
    std::vector<Id> queue{entry_point_};
    seen[entry_point_] = true;
    for (std::size_t i = 0; i < queue.size(); ++i) {
        for (const Id id : links(queue[i], 0)) {
            if (id < n && !seen[id]) {
                seen[id] = true;
                queue.push_back(id);
            }
        }
    }
    r.reachable = queue.size();
    r.mean_degree0 = static_cast<double>(degree0) / static_cast<double>(n);
    return r;
}

}  // namespace vdx
