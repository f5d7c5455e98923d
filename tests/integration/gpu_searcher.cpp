// The vecdex-side binding shown in INTEGRATION.md ("The C ABI, from inside vecdex"), compiled the
// way a vecdex maintainer would compile it: against the reference's own headers
// (include/vecdex/hnsw.hpp, matrix.hpp, neighbor.hpp) and include/vdx_b200.h, linked with the
// reference library and libvdx_b200.so.
//
//   gpu_searcher <index.vdx> <queries.f32> <nq> <dim> <k> <ef>
//
// Loads the index with both libraries, runs the queries (nq x dim raw float32) through
// GpuSearcher::search_batch and through vecdex::HnswIndex::search_batch
// (include/vecdex/hnsw.hpp:97), and exits 0 when every result list is the same (ids and distance
// bits), 1 when one differs, 2 on an error (the message on stderr). Test program: built by
// oracle/Makefile (target `integration`) into oracle/_ref/, run by tests/test_integration.py.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <span>
#include <stdexcept>
#include <vector>

#include "vdx_b200.h"
#include "vecdex/hnsw.hpp"

namespace vecdex {

class GpuSearcher {
public:
    // The device copy is built from the same file vecdex saved (docs/FORMAT.md v1).
    explicit GpuSearcher(const std::filesystem::path& saved) {
        check(vdx_index_load(saved.c_str(), &h_));
        check(vdx_index_upload(h_, /*device=*/0, VDX_FP32));
    }
    ~GpuSearcher() { vdx_index_free(h_); }
    GpuSearcher(const GpuSearcher&) = delete;
    GpuSearcher& operator=(const GpuSearcher&) = delete;

    // Same contract as HnswIndex::search_batch (include/vecdex/hnsw.hpp:97).
    std::vector<std::vector<Neighbor>> search_batch(MatrixView<float> q, std::size_t k,
                                                    std::size_t ef) const {
        std::vector<uint32_t> ids(q.rows() * k), counts(q.rows());
        std::vector<float> d(q.rows() * k);
        check(vdx_search_batch(h_, q.data().data(), q.rows(), q.dim(), k, ef, ids.data(),
                               d.data(), counts.data(), nullptr));
        std::vector<std::vector<Neighbor>> out(q.rows());
        for (std::size_t r = 0; r < q.rows(); ++r) {
            for (uint32_t i = 0; i < counts[r]; ++i) {
                out[r].push_back({d[r * k + i], ids[r * k + i]});
            }
        }
        return out;
    }

private:
    static void check(vdx_status s) {
        if (s == VDX_ERR_INVALID_ARGUMENT) throw std::invalid_argument(vdx_last_error());
        if (s == VDX_ERR_LENGTH) throw std::length_error(vdx_last_error());
        if (s != VDX_OK) throw std::runtime_error(vdx_last_error());
    }
    vdx_index* h_ = nullptr;
};

}  // namespace vecdex

int main(int argc, char** argv) {
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s index.vdx queries.f32 nq dim k ef\n", argv[0]);
        return 2;
    }
    try {
        const std::size_t nq = std::strtoull(argv[3], nullptr, 10);
        const std::size_t dim = std::strtoull(argv[4], nullptr, 10);
        const std::size_t k = std::strtoull(argv[5], nullptr, 10);
        const std::size_t ef = std::strtoull(argv[6], nullptr, 10);
        std::vector<float> q(nq * dim);
        std::ifstream in(argv[2], std::ios::binary);
        if (!in.read(reinterpret_cast<char*>(q.data()), static_cast<std::streamsize>(q.size() * 4))) {
            throw std::runtime_error("cannot read the query file");
        }
        const vecdex::MatrixView<float> view(std::span<const float>(q), dim);
        const vecdex::GpuSearcher gpu(argv[1]);
        const auto got = gpu.search_batch(view, k, ef);
        const auto ref = vecdex::HnswIndex::load(argv[1]);
        const auto want = ref.search_batch(view, k, ef);
        std::size_t differ = 0;
        for (std::size_t r = 0; r < nq; ++r) {
            bool same = got[r].size() == want[r].size();
            for (std::size_t i = 0; same && i < got[r].size(); ++i) {
                same = got[r][i].id == want[r][i].id &&
                       std::memcmp(&got[r][i].distance, &want[r][i].distance, 4) == 0;
            }
            differ += same ? 0 : 1;
        }
        std::printf("queries %zu differing %zu\n", nq, differ);
        return differ == 0 ? 0 : 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 2;
    }
}
