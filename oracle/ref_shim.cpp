// TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A C-ABI shim over the unmodified vecdex reference library (compiled from its own sources by
// oracle/Makefile into oracle/_ref/libvecdex_ref.so). Only the tests, the smoke check and
// bench.py's CPU-baseline / reference arm load it: it is the checker and the timed CPU baseline,
// never part of the GPU product path.
//
// Every function calls the reference's public C++ API and nothing else:
//   HnswIndex(dim, metric, params), add(MatrixView, threads)   include/vecdex/hnsw.hpp:67,87
//   HnswIndex::search / search_batch                            include/vecdex/hnsw.hpp:93,97
//   HnswIndex::save / load / inspect                            include/vecdex/hnsw.hpp:102-123
//   BruteForceIndex(dim, metric), add, search                   include/vecdex/brute_force.hpp:21-36
//   kernels::active()                                           include/vecdex/kernels.hpp:31
// Exceptions never cross the ABI: each call returns 0 on success, or a negative code with the
// message kept for vref_last_error().

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "vecdex/brute_force.hpp"
#include "vecdex/distance.hpp"
#include "vecdex/hnsw.hpp"
#include "vecdex/kernels.hpp"
#include "vecdex/matrix.hpp"

namespace {

thread_local std::string g_last_error;

vecdex::Metric metric_of(int code) {
    switch (code) {
        case 0:
            return vecdex::Metric::L2;
        case 1:
            return vecdex::Metric::InnerProduct;
        case 2:
            return vecdex::Metric::Cosine;
        default:
            throw std::invalid_argument("unknown metric code");
    }
}

int metric_code(vecdex::Metric m) {
    switch (m) {
        case vecdex::Metric::L2:
            return 0;
        case vecdex::Metric::InnerProduct:
            return 1;
        case vecdex::Metric::Cosine:
            return 2;
    }
    return -1;
}

// -1 invalid_argument, -2 length_error, -3 runtime_error (I/O), -4 anything else.
template <typename Fn>
int guarded(Fn&& fn) {
    try {
        fn();
        return 0;
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return -1;
    } catch (const std::length_error& e) {
        g_last_error = e.what();
        return -2;
    } catch (const std::runtime_error& e) {
        g_last_error = e.what();
        return -3;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -4;
    }
}

void write_results(const std::vector<vecdex::Neighbor>& found, std::size_t k, std::uint32_t* ids,
                   float* dists, std::uint32_t* count) {
    for (std::size_t i = 0; i < k; ++i) {
        if (i < found.size()) {
            ids[i] = found[i].id;
            dists[i] = found[i].distance;
        } else {
            ids[i] = 0xFFFFFFFFU;
            dists[i] = __builtin_inff();
        }
    }
    *count = static_cast<std::uint32_t>(found.size());
}

std::size_t resolve(std::size_t threads) {
    return threads != 0 ? threads : std::max(1U, std::thread::hardware_concurrency());
}

}  // namespace

extern "C" {

const char* vref_last_error() { return g_last_error.c_str(); }

const char* vref_isa() {
    static const std::string name(vecdex::kernels::name(vecdex::kernels::active().isa));
    return name.c_str();
}

float vref_l2(const float* a, const float* b, std::uint64_t dim) {
    return vecdex::kernels::active().l2_squared(a, b, dim);
}

float vref_ip(const float* a, const float* b, std::uint64_t dim) {
    return vecdex::kernels::active().inner_product(a, b, dim);
}

int vref_hnsw_new(std::uint64_t dim, int metric, std::uint64_t M, std::uint64_t ef_construction,
                  std::uint64_t seed, void** out) {
    return guarded([&] {
        auto index = std::make_unique<vecdex::HnswIndex>(
            dim, metric_of(metric),
            vecdex::HnswParams{.M = M, .ef_construction = ef_construction, .seed = seed});
        *out = index.release();
    });
}

void vref_hnsw_free(void* h) { delete static_cast<vecdex::HnswIndex*>(h); }

// add(MatrixView, threads): threads = 1 is the deterministic serial build.
int vref_hnsw_add(void* h, const float* data, std::uint64_t rows, std::uint64_t dim,
                  std::uint64_t threads) {
    return guarded([&] {
        auto* index = static_cast<vecdex::HnswIndex*>(h);
        index->add(vecdex::MatrixView<float>(std::span<const float>(data, rows * dim), dim),
                   threads);
    });
}

// add(span) one vector at a time: the "one_by_one" build of the reference's fingerprint test.
int vref_hnsw_add_one(void* h, const float* v, std::uint64_t dim, std::uint32_t* id) {
    return guarded([&] {
        auto* index = static_cast<vecdex::HnswIndex*>(h);
        *id = index->add(std::span<const float>(v, dim));
    });
}

int vref_hnsw_save(void* h, const char* path) {
    return guarded([&] { static_cast<vecdex::HnswIndex*>(h)->save(path); });
}

int vref_hnsw_load(const char* path, void** out) {
    return guarded([&] {
        auto index = std::make_unique<vecdex::HnswIndex>(vecdex::HnswIndex::load(path));
        *out = index.release();
    });
}

void vref_hnsw_info(void* h, std::uint64_t* size, std::uint64_t* dim, int* metric,
                    std::uint64_t* M, std::uint64_t* memory_bytes) {
    auto* index = static_cast<vecdex::HnswIndex*>(h);
    *size = index->size();
    *dim = index->dim();
    *metric = metric_code(index->metric());
    *M = index->params().M;
    *memory_bytes = index->memory_bytes();
}

// inspect(): violations count, reachable, max_level, mean_degree0.
int vref_hnsw_inspect(void* h, std::uint64_t* violations, std::uint64_t* reachable,
                      std::uint64_t* max_level, double* mean_degree0) {
    return guarded([&] {
        const vecdex::GraphReport r = static_cast<vecdex::HnswIndex*>(h)->inspect();
        *violations = r.violations.size();
        *reachable = r.reachable;
        *max_level = r.max_level;
        *mean_degree0 = r.mean_degree0;
    });
}

// search(): one query on the calling thread.
int vref_hnsw_search(void* h, const float* q, std::uint64_t dim, std::uint64_t k, std::uint64_t ef,
                     std::uint32_t* ids, float* dists, std::uint32_t* count) {
    return guarded([&] {
        auto* index = static_cast<vecdex::HnswIndex*>(h);
        write_results(index->search(std::span<const float>(q, dim), k, ef), k, ids, dists, count);
    });
}

// search_batch(): results padded to k per row (id 0xFFFFFFFF, distance +inf), count per row.
int vref_hnsw_search_batch(void* h, const float* queries, std::uint64_t nq, std::uint64_t dim,
                           std::uint64_t k, std::uint64_t ef, std::uint64_t threads,
                           std::uint32_t* ids, float* dists, std::uint32_t* counts) {
    return guarded([&] {
        auto* index = static_cast<vecdex::HnswIndex*>(h);
        const auto found = index->search_batch(
            vecdex::MatrixView<float>(std::span<const float>(queries, nq * dim), dim), k, ef,
            threads);
        for (std::size_t q = 0; q < found.size(); ++q) {
            write_results(found[q], k, ids + q * k, dists + q * k, counts + q);
        }
    });
}

// search_batch() timed like bench/hnsw_eval.cpp:493-512 (one warm-up pass, then `repeats`
// passes); returns every pass's wall time in seconds, so the caller can take the median.
int vref_hnsw_time_search_batch(void* h, const float* queries, std::uint64_t nq,
                                std::uint64_t dim, std::uint64_t k, std::uint64_t ef,
                                std::uint64_t threads, std::uint64_t repeats, double* seconds) {
    return guarded([&] {
        auto* index = static_cast<vecdex::HnswIndex*>(h);
        const vecdex::MatrixView<float> view(std::span<const float>(queries, nq * dim), dim);
        (void)index->search_batch(view, k, ef, threads);
        for (std::uint64_t r = 0; r < repeats; ++r) {
            const auto start = std::chrono::steady_clock::now();
            const auto found = index->search_batch(view, k, ef, threads);
            seconds[r] =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        }
    });
}

int vref_bf_new(std::uint64_t dim, int metric, void** out) {
    return guarded([&] {
        auto index = std::make_unique<vecdex::BruteForceIndex>(dim, metric_of(metric));
        *out = index.release();
    });
}

void vref_bf_free(void* h) { delete static_cast<vecdex::BruteForceIndex*>(h); }

int vref_bf_add(void* h, const float* data, std::uint64_t rows, std::uint64_t dim) {
    return guarded([&] {
        vecdex::Matrix<float> m(rows, dim);
        std::memcpy(m.data().data(), data, rows * dim * sizeof(float));
        static_cast<vecdex::BruteForceIndex*>(h)->add(m);
    });
}

// BruteForceIndex::search for every row, parallelized over queries with the claim-counter
// scheme of bench/hnsw_eval.cpp:77-103 (the reference has no batch API for brute force).
int vref_bf_search_batch(void* h, const float* queries, std::uint64_t nq, std::uint64_t dim,
                         std::uint64_t k, std::uint64_t threads, std::uint32_t* ids, float* dists,
                         std::uint32_t* counts) {
    return guarded([&] {
        auto* index = static_cast<const vecdex::BruteForceIndex*>(h);
        std::atomic<std::uint64_t> next{0};
        std::exception_ptr error;
        std::atomic<bool> failed{false};
        const auto work = [&] {
            try {
                for (std::uint64_t q = next.fetch_add(1); q < nq; q = next.fetch_add(1)) {
                    write_results(index->search(std::span<const float>(queries + q * dim, dim), k),
                                  k, ids + q * k, dists + q * k, counts + q);
                }
            } catch (...) {
                next.store(nq);
                if (!failed.exchange(true)) {
                    error = std::current_exception();
                }
            }
        };
        std::vector<std::thread> helpers;
        const std::size_t t = std::min<std::size_t>(resolve(threads), std::max<std::uint64_t>(nq, 1));
        for (std::size_t i = 1; i < t; ++i) {
            helpers.emplace_back(work);
        }
        work();
        for (auto& th : helpers) {
            th.join();
        }
        if (error) {
            std::rethrow_exception(error);
        }
    });
}

}  // extern "C"
