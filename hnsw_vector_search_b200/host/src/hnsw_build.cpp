// HnswIndex construction and diagnostics on the host.
//
// The graph must be the one the reference builds (src/hnsw.cpp:223-409 of the reference), so that
// serial builds agree byte for byte and GPU results can be compared id for id: the level draw
// (top 53 bits of mt19937_64, floor(-ln U / ln M)), the insertion procedure (greedy descent,
// per-layer candidate search with ef = max(ef_construction, M), neighbor selection, links back)
// and the selection heuristic are the same steps in the same order. The code is this project's
// own. Parallel add() uses one lock per node, held one at a time, so no lock cycle can form.

#include <algorithm>
#include <atomic>
#include <cassert>
#include <cmath>
#include <exception>
#include <format>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <utility>

#include "internal.hpp"
#include "vdx/device.hpp"
#include "vdx/hnsw.hpp"

namespace vdx {

struct HnswIndex::BuildLocks {
    explicit BuildLocks(std::size_t n) : node(std::make_unique<std::mutex[]>(n)) {}
    std::unique_ptr<std::mutex[]> node;  // guards that node's link blocks on every layer
    std::mutex entry;                    // guards entry_point_ and max_level_
};

// Per-insert scratch: visited stamps and the two heaps of the layer search.
struct BuildScratch {
    std::vector<std::uint32_t> stamp;
    std::uint32_t epoch = 0;
    std::vector<Neighbor> frontier;  // heap, closest on top
    std::vector<Neighbor> best;      // heap, worst on top
    std::vector<Id> fresh;
    std::vector<Id> copy;

    void begin(std::size_t n) {
        if (stamp.size() < n) {
            stamp.resize(n, 0);
        }
        if (++epoch == 0) {
            std::ranges::fill(stamp, 0U);
            epoch = 1;
        }
    }
    bool first_visit(Id id) noexcept {
        if (stamp[id] == epoch) {
            return false;
        }
        stamp[id] = epoch;
        return true;
    }
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

// Heap orders for std heaps (greatest on top): `frontier` keeps the closest on top,
// `best` keeps the worst on top.
bool frontier_order(const Neighbor& a, const Neighbor& b) noexcept { return closer(b, a); }
bool best_order(const Neighbor& a, const Neighbor& b) noexcept { return closer(a, b); }

std::size_t thread_count(std::size_t requested) noexcept {
    return requested != 0 ? requested : std::max(1U, std::thread::hardware_concurrency());
}

// fn(i) for i in [0, count) on `threads` threads claiming items from a shared counter; the first
// exception is rethrown after all threads stop.
template <typename Fn>
void run_parallel(std::size_t count, std::size_t threads, const Fn& fn) {
    if (count == 0) {
        return;
    }
    std::atomic<std::size_t> next{0};
    std::exception_ptr error;
    std::mutex error_lock;
    const auto worker = [&] {
        try {
            for (std::size_t i = next++; i < count; i = next++) {
                fn(i);
            }
        } catch (...) {
            next = count;
            const std::scoped_lock lock(error_lock);
            if (!error) {
                error = std::current_exception();
            }
        }
    };
    std::vector<std::thread> pool;
    for (std::size_t t = 1; t < std::min(threads, count); ++t) {
        try {
            pool.emplace_back(worker);
        } catch (...) {
            break;  // fewer threads: the work still gets done
        }
    }
    worker();
    for (auto& t : pool) {
        t.join();
    }
    if (error) {
        std::rethrow_exception(error);
    }
}

}  // namespace

HnswIndex::HnswIndex(std::size_t dim, Metric metric, HnswParams params)
    : metric_(metric),
      params_(validated(params)),
      level_multiplier_(1.0 / std::log(static_cast<double>(params_.M))),
      rng_(params_.seed),
      vectors_(dim),
      device_mutex_(std::make_unique<std::mutex>()) {}

HnswIndex::~HnswIndex() = default;
HnswIndex::HnswIndex(HnswIndex&&) noexcept = default;
HnswIndex& HnswIndex::operator=(HnswIndex&&) noexcept = default;

const Id* HnswIndex::link_block(Id node, std::size_t layer) const noexcept {
    if (layer == 0) {
        return layer0_.data() + static_cast<std::size_t>(node) * (1 + max_links(0));
    }
    return upper_[node].data() + (layer - 1) * (1 + max_links(layer));
}

Id* HnswIndex::link_block(Id node, std::size_t layer) noexcept {
    return const_cast<Id*>(std::as_const(*this).link_block(node, layer));
}

std::span<const Id> HnswIndex::links(Id node, std::size_t layer) const noexcept {
    const Id* block = link_block(node, layer);
    return {block + 1, block[0]};
}

void HnswIndex::set_links(Id node, std::size_t layer, std::span<const Neighbor> chosen) noexcept {
    Id* block = link_block(node, layer);
    block[0] = static_cast<Id>(chosen.size());
    for (std::size_t i = 0; i < chosen.size(); ++i) {
        block[1 + i] = chosen[i].id;
    }
}

float HnswIndex::dist(const float* a, const float* b) const noexcept {
    if (metric_ == Metric::L2) {
        return detail::l2_squared_raw(a, b, dim());
    }
    return 1.0F - detail::inner_product_raw(a, b, dim());
}

std::size_t HnswIndex::memory_bytes() const noexcept {
    // Every node's upper vector holds exactly level x (1 + M) ids (store() and load() size them
    // so), which lets the levels give the total without visiting n separate allocations.
    std::size_t blocks = 0;
    for (const std::uint8_t level : levels_) {
        blocks += level;
    }
    return vectors_.data().size_bytes() + levels_.size() + layer0_.size() * sizeof(Id) +
           upper_.size() * sizeof(std::vector<Id>) + blocks * (1 + max_links(1)) * sizeof(Id);
}

void HnswIndex::invalidate_device() noexcept {
    if (device_mutex_) {
        const std::scoped_lock lock(*device_mutex_);
        device_.clear();
    }
}

// U = 1 - (top 53 bits) * 2^-53 lies in (0, 1]; level = floor(-ln U * mL).
std::size_t HnswIndex::random_level() {
    const double u = 1.0 - static_cast<double>(rng_() >> 11U) * 0x1.0p-53;
    return static_cast<std::size_t>(-std::log(u) * level_multiplier_);
}

void HnswIndex::store(std::span<const float> vector) {
    if (!device_mutex_) {  // moved-from index being reused
        device_mutex_ = std::make_unique<std::mutex>();
    }
    vectors_.append(vector);
    if (metric_ == Metric::Cosine) {
        detail::normalize(vectors_.row(size() - 1));
    }
    const std::size_t level = random_level();
    levels_.push_back(static_cast<std::uint8_t>(level));
    layer0_.resize(layer0_.size() + 1 + max_links(0), Id{0});
    upper_.emplace_back(level * (1 + max_links(1)), Id{0});
}

Id HnswIndex::add(std::span<const float> vector) {
    detail::check_new_vectors("HnswIndex::add", {metric_, dim(), size()}, vector.size(), vector);
    invalidate_device();
    store(vector);
    const auto id = static_cast<Id>(size() - 1);
    insert<Locking::None>(id);
    return id;
}

void HnswIndex::add(const Matrix<float>& vectors, std::size_t num_threads) {
    add(MatrixView<float>(vectors), num_threads);
}

void HnswIndex::add(MatrixView<float> vectors, std::size_t num_threads) {
    detail::check_new_vectors("HnswIndex::add", {metric_, dim(), size()}, vectors.dim(),
                              vectors.data());
    invalidate_device();
    const std::size_t first = size();
    const std::size_t total = first + vectors.rows();
    vectors_.reserve_rows(total);
    levels_.reserve(total);
    layer0_.reserve(total * (1 + max_links(0)));
    upper_.reserve(total);
    const std::size_t threads = std::min(thread_count(num_threads), vectors.rows());
    if (threads <= 1) {
        for (std::size_t r = 0; r < vectors.rows(); ++r) {
            store(vectors.row(r));
            insert<Locking::None>(static_cast<Id>(size() - 1));
        }
        return;
    }
    // Every vector is stored (levels drawn in serial order) before any is linked, so no container
    // grows while other threads read it.
    build_locks_ = std::make_unique<BuildLocks>(total);
    for (std::size_t r = 0; r < vectors.rows(); ++r) {
        store(vectors.row(r));
    }
    std::size_t next = first;
    if (next == 0) {
        insert<Locking::None>(0);
        next = 1;
    }
    run_parallel(total - next, threads,
                 [this, next](std::size_t i) { insert<Locking::PerNode>(static_cast<Id>(next + i)); });
    build_locks_.reset();
}

template <HnswIndex::Locking L>
std::span<const Id> HnswIndex::read_links(Id node, std::size_t layer,
                                          std::vector<Id>& copy) const {
    if constexpr (L == Locking::PerNode) {
        const std::scoped_lock lock(build_locks_->node[node]);
        const auto ids = links(node, layer);
        copy.assign(ids.begin(), ids.end());
        return copy;
    } else {
        return links(node, layer);
    }
}

template <HnswIndex::Locking L>
Neighbor HnswIndex::build_greedy(const float* query, Neighbor entry, std::size_t layer,
                                 std::vector<Id>& copy) const {
    bool moved = true;
    while (moved) {
        moved = false;
        for (const Id id : read_links<L>(entry.id, layer, copy)) {
            const float d = dist(query, vector_of(id));
            if (d < entry.distance) {
                entry = {d, id};
                moved = true;
            }
        }
    }
    return entry;
}

template <HnswIndex::Locking L>
void HnswIndex::build_search_layer(const float* query, Neighbor entry, std::size_t ef,
                                   std::size_t layer, BuildScratch& s) const {
    s.begin(size());
    s.first_visit(entry.id);
    s.frontier.assign(1, entry);
    s.best.assign(1, entry);
    while (!s.frontier.empty()) {
        std::ranges::pop_heap(s.frontier, frontier_order);
        const Neighbor current = s.frontier.back();
        s.frontier.pop_back();
        if (s.best.size() >= ef && closer(s.best.front(), current)) {
            break;
        }
        s.fresh.clear();
        for (const Id id : read_links<L>(current.id, layer, s.copy)) {
            if (s.first_visit(id)) {
                s.fresh.push_back(id);
            }
        }
        for (const Id id : s.fresh) {
            const Neighbor n{dist(query, vector_of(id)), id};
            if (s.best.size() < ef || closer(n, s.best.front())) {
                s.frontier.push_back(n);
                std::ranges::push_heap(s.frontier, frontier_order);
                s.best.push_back(n);
                std::ranges::push_heap(s.best, best_order);
                if (s.best.size() > ef) {
                    std::ranges::pop_heap(s.best, best_order);
                    s.best.pop_back();
                }
            }
        }
    }
}

template <HnswIndex::Locking L>
void HnswIndex::insert(Id node) {
    const std::size_t level = levels_[node];
    if (node == 0) {
        entry_point_ = 0;
        max_level_ = level;
        return;
    }
    std::unique_lock<std::mutex> entry_lock;
    if constexpr (L == Locking::PerNode) {
        entry_lock = std::unique_lock(build_locks_->entry);
    }
    const Id entry_point = entry_point_;
    const std::size_t max_level = max_level_;
    if (entry_lock.owns_lock() && level <= max_level) {
        entry_lock.unlock();  // only a node raising the top layer keeps it
    }
    thread_local BuildScratch scratch;
    const float* query = vector_of(node);
    Neighbor entry{dist(query, vector_of(entry_point)), entry_point};
    for (std::size_t layer = max_level; layer > level; --layer) {
        entry = build_greedy<L>(query, entry, layer, scratch.copy);
    }
    const std::size_t ef = std::max(params_.ef_construction, params_.M);
    const std::size_t top = std::min(level, max_level);
    std::vector<std::vector<Neighbor>> chosen(top + 1);
    for (std::size_t i = 0; i <= top; ++i) {
        const std::size_t layer = top - i;
        build_search_layer<L>(query, entry, ef, layer, scratch);
        entry = *std::ranges::min_element(scratch.best, closer);
        chosen[layer] = select_neighbors(scratch.best, params_.M);
    }
    {
        std::unique_lock<std::mutex> own;
        if constexpr (L == Locking::PerNode) {
            own = std::unique_lock(build_locks_->node[node]);
        }
        for (std::size_t layer = 0; layer <= top; ++layer) {
            set_links(node, layer, chosen[layer]);
        }
    }
    for (std::size_t layer = 0; layer <= top; ++layer) {
        link_back<L>(node, layer, chosen[layer]);
    }
    if (level > max_level) {
        max_level_ = level;
        entry_point_ = node;
    }
}

template <HnswIndex::Locking L>
void HnswIndex::link_back(Id node, std::size_t layer, std::span<const Neighbor> chosen) {
    for (const Neighbor& n : chosen) {
        std::unique_lock<std::mutex> lock;
        if constexpr (L == Locking::PerNode) {
            lock = std::unique_lock(build_locks_->node[n.id]);
        }
        Id* block = link_block(n.id, layer);
        const std::size_t count = block[0];
        if (count < max_links(layer)) {
            block[1 + count] = node;
            block[0] = static_cast<Id>(count + 1);
            continue;
        }
        std::vector<Neighbor> candidates;
        candidates.reserve(count + 1);
        const float* base = vector_of(n.id);
        for (const Id id : links(n.id, layer)) {
            candidates.push_back({dist(base, vector_of(id)), id});
        }
        candidates.push_back({n.distance, node});
        set_links(n.id, layer, select_neighbors(std::move(candidates), max_links(layer)));
    }
}

// Keep a candidate (closest first) only if it is closer to the base node than to every
// candidate already kept; with m or fewer candidates keep all.
std::vector<Neighbor> HnswIndex::select_neighbors(std::vector<Neighbor> candidates,
                                                  std::size_t m) const {
    std::ranges::sort(candidates, closer);
    if (candidates.size() <= m) {
        return candidates;
    }
    std::vector<Neighbor> kept;
    kept.reserve(m);
    for (const Neighbor& c : candidates) {
        if (kept.size() == m) {
            break;
        }
        const float* v = vector_of(c.id);
        bool diverse = true;
        for (const Neighbor& k : kept) {
            if (dist(v, vector_of(k.id)) < c.distance) {
                diverse = false;
                break;
            }
        }
        if (diverse) {
            kept.push_back(c);
        }
    }
    return kept;
}

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
