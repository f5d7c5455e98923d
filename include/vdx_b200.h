/*
 * vdx_b200: the C ABI of the B200 batched query path for vecdex HNSW indexes.
 *
 * This is the drop-in boundary. Every entry point takes plain pointers and sizes, returns a
 * vdx_status, and never lets a C++ exception cross it; the message of the last failure on the
 * calling thread is vdx_last_error(). Each function names the reference interface it replaces
 * (paths inside the vecdex reference project, MatiiiBL/HNSW_vector_search). Error classes map to
 * the reference's exception types: VDX_ERR_INVALID_ARGUMENT = std::invalid_argument (with the
 * reference's messages), VDX_ERR_LENGTH = std::length_error, VDX_ERR_IO = std::runtime_error
 * from save/load (message starting with the path).
 *
 * Threading: as in the reference (include/vecdex/hnsw.hpp:58-62), searches may run
 * concurrently from several threads, but not concurrently with vdx_index_add.
 * Ownership: handles own all their storage (host and device); callers own every buffer they pass.
 */
#ifndef VDX_B200_H
#define VDX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VDX_API __attribute__((visibility("default")))

typedef enum vdx_status {
    VDX_OK = 0,
    VDX_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
    VDX_ERR_LENGTH = 2,           /* std::length_error */
    VDX_ERR_IO = 3,               /* std::runtime_error from save / load */
    VDX_ERR_CUDA = 4,             /* a CUDA call failed, or no device is present */
    VDX_ERR_INTERNAL = 5,
    /* No reference counterpart (the reference has no device code). A bounded device wait gave up
     * (the tensor-core brute force's pipeline barriers): the kernel drained its own copies and
     * tensor-core work, freed its tensor memory and returned, so the context stays usable and
     * the next call may be retried. */
    VDX_ERR_DEVICE_TIMEOUT = 6,
    /* No reference counterpart. A kernel met a link id outside the index in the device copy of
     * the graph (a corrupted device mirror); the access was skipped. */
    VDX_ERR_DEVICE_BOUNDS = 7
} vdx_status;

/* Metric codes are the file format's (docs/FORMAT.md "Header"): 0 L2, 1 inner product, 2 cosine. */
enum { VDX_METRIC_L2 = 0, VDX_METRIC_IP = 1, VDX_METRIC_COSINE = 2 };
/* Traversal precision of the GPU search. */
enum { VDX_FP32 = 0, VDX_BF16 = 1, VDX_FP8 = 2 };
/* Brute-force scoring method. */
enum { VDX_BF_EXACT = 0, VDX_BF_TENSOR_CORE = 1 };

typedef struct vdx_index vdx_index;
typedef struct vdx_bruteforce vdx_bruteforce;

typedef struct vdx_index_info {
    uint64_t size, dim, M, ef_construction, seed, max_level, entry_point, memory_bytes;
    uint32_t metric;
} vdx_index_info;

typedef struct vdx_graph_report {
    uint64_t violations, reachable, max_level;
    double mean_degree0;
} vdx_graph_report;

typedef struct vdx_search_options {
    uint32_t precision;      /* VDX_FP32 (reference-identical results), VDX_BF16, VDX_FP8 */
    uint32_t rerank;         /* BF16 / FP8: candidates re-scored in FP32; 0 = 4k, 0xFFFFFFFF = none */
    uint32_t learned_stop;   /* nonzero: learned early termination (needs a model) */
    float stop_threshold;    /* stop when the network's "converged" probability reaches this */
    int32_t device;
    uint32_t stop_gate;      /* learned stop: consult the network at a checkpoint only once the k-th
                                distance has been unchanged for this many expansions in a row
                                (0 to 3; 0 = at every checkpoint) */
} vdx_search_options;

/* Statistics words of a search (vdx_last_stats, vdx_search_batch_device). */
enum {
    VDX_STAT_QUERIES = 0, VDX_STAT_EXPANSIONS, VDX_STAT_DIST_LAYER0, VDX_STAT_DIST_UPPER,
    VDX_STAT_LINK_BYTES, VDX_STAT_ROW_BYTES, VDX_STAT_RERANK_BYTES, VDX_STAT_DUPLICATES,
    VDX_STAT_PREFETCH_HITS, VDX_STAT_LEARNED_STOPS, VDX_STAT_COUNT,
    /* after a brute-force batch: queries the tensor-core path could not certify */
    VDX_STAT_BF_UNCERTIFIED = 12
};

VDX_API const char* vdx_last_error(void);
VDX_API const char* vdx_version(void);
VDX_API int vdx_device_count(void);

/* --- HnswIndex lifecycle (host) ------------------------------------------------------------ */

/* HnswIndex(dim, metric, {M, ef_construction, seed}): include/vecdex/hnsw.hpp:67 */
VDX_API vdx_status vdx_index_create(uint64_t dim, uint32_t metric, uint64_t M,
                                    uint64_t ef_construction, uint64_t seed, vdx_index** out);
VDX_API void vdx_index_free(vdx_index* index);
/* add(MatrixView<float>, num_threads): include/vecdex/hnsw.hpp:87 (num_threads 1 = the serial,
 * reproducible build; 0 = one thread per hardware thread) */
VDX_API vdx_status vdx_index_add(vdx_index* index, const float* rows, uint64_t n, uint64_t dim,
                                 uint64_t num_threads);
/* vdx_index_add built on the GPU (device): batched parallel insertion whose graph matches a
 * parallel build's quality (recall within 0.005 of the serial build), the levels drawn in the
 * serial order. Replaces the reference's HnswIndex::add(vectors, threads) for large batches
 * (src/hnsw.cpp:270-290); same validation and errors. */
VDX_API vdx_status vdx_index_add_gpu(vdx_index* index, const float* data, uint64_t rows, uint64_t dim,
                                     int32_t device);
/* add(span<const float>): include/vecdex/hnsw.hpp:80 */
VDX_API vdx_status vdx_index_add_one(vdx_index* index, const float* vector, uint64_t dim,
                                     uint32_t* id);
/* save(path): include/vecdex/hnsw.hpp:115 */
VDX_API vdx_status vdx_index_save(const vdx_index* index, const char* path);
/* load(path): include/vecdex/hnsw.hpp:123 */
VDX_API vdx_status vdx_index_load(const char* path, vdx_index** out);
/* No reference counterpart (the reference has no device mirror). The FP32 device mirror as a
 * sidecar file next to the v1 index file: a 4096-byte header, then the device arrays (FP32 rows
 * padded to 16 bytes, layer-0 blocks, upper-block index, upper blocks), each section 4096-byte
 * aligned. save writes it on the host; load installs it as the FP32 mirror of `device` with one
 * copy per section and fails (VDX_ERR_IO) if the file names another graph (its XXH64 of the
 * vectors, levels and link blocks differs), is truncated or is not a device image. */
VDX_API vdx_status vdx_index_save_device_image(const vdx_index* index, const char* path);
VDX_API vdx_status vdx_index_load_device_image(const vdx_index* index, const char* path,
                                               int32_t device);
/* No reference counterpart: the XXH64 a device image names its graph by (the vectors, the
 * levels, the layer-0 blocks and the upper blocks of the v1 layout, hashed in that order). */
VDX_API vdx_status vdx_index_graph_hash(const vdx_index* index, uint64_t* out);
/* size() / dim() / metric() / params() / memory_bytes(): include/vecdex/hnsw.hpp:74-77,105 */
VDX_API vdx_status vdx_index_info_get(const vdx_index* index, vdx_index_info* out);
/* inspect(): include/vecdex/hnsw.hpp:102; the first violation's text is copied into `first`
 * (capacity `cap` bytes, may be NULL) */
VDX_API vdx_status vdx_index_inspect(const vdx_index* index, vdx_graph_report* out, char* first,
                                     uint64_t cap);

/* --- HNSW search on the GPU -------------------------------------------------------------- */

/* search_batch(queries, k, ef): include/vecdex/hnsw.hpp:97 (src/hnsw.cpp:490-501).
 * Host buffers: queries nq x dim; ids, dists nq x k (rows shorter than k padded with
 * 0xFFFFFFFF / +inf); counts nq. Synchronous. opts may be NULL (FP32, device 0). */
VDX_API vdx_status vdx_search_batch(const vdx_index* index, const float* queries, uint64_t nq,
                                    uint64_t dim, uint64_t k, uint64_t ef, uint32_t* ids,
                                    float* dists, uint32_t* counts,
                                    const vdx_search_options* opts);
/* search(query, k, ef): include/vecdex/hnsw.hpp:93; `ids`/`dists` hold k entries. */
VDX_API vdx_status vdx_search(const vdx_index* index, const float* query, uint64_t dim,
                              uint64_t k, uint64_t ef, uint32_t* ids, float* dists,
                              uint32_t* count);
/* The statistics words (VDX_STAT_*) of this thread's last vdx_search_batch. */
VDX_API vdx_status vdx_last_stats(uint64_t* out, uint64_t count);

/* Builds (or refreshes after add) the device mirror for (device, precision) now, so that the
 * first search does not pay for the upload. */
VDX_API vdx_status vdx_index_upload(const vdx_index* index, int32_t device, uint32_t precision);

/* Device-resident batch, asynchronous on `stream` (a cudaStream_t, or NULL for the legacy
 * default stream): the kernel-only form of vdx_search_batch for callers whose queries and
 * results live in device memory. Per-query k and ef come from d_k / d_ef when not NULL, else
 * k_uniform / ef_uniform; result rows are out_stride wide (without d_k, out_stride must be at
 * least k_uniform; with d_k, a row's count is cut to out_stride; each d_ef[i] must fit the result
 * capacity the uniform ef sets, the next power of two >= max(ef_uniform, 32), else that row
 * reports code 4). d_work is caller-owned device memory
 * of vdx_work_words() u32 words: [0] error code (0 = ok; 1 non-finite query, 2 zero cosine
 * query, 3 corrupt device graph, 4 ef above capacity), [1] the lowest failing row, [16..] the
 * 64-bit statistics words. The call does not wait for the kernel. The search runs as three
 * kernels (an upper-layer descent for every query, a one-block ordering of the queries by their
 * layer-0 entry distance, the layer-0 searches, farthest entries first so the costliest start
 * first), with 12 bytes per query of scratch taken from and returned to a library-owned
 * stream-ordered pool on `stream`. */
VDX_API uint64_t vdx_work_words(void);
/* Kernels the calling thread's last HNSW search launched (3 for the ordered search above and
 * vdx_search_batch, 1 for vdx_search_batch_device_noalloc), for launch accounting. */
VDX_API uint32_t vdx_search_kernels_last(void);
VDX_API vdx_status vdx_search_batch_device(const vdx_index* index, const float* d_queries,
                                           uint64_t nq, uint64_t dim, const uint32_t* d_k,
                                           const uint32_t* d_ef, uint32_t k_uniform,
                                           uint32_t ef_uniform, uint32_t out_stride,
                                           uint32_t* d_ids, float* d_dists, uint32_t* d_counts,
                                           uint32_t* d_work, const vdx_search_options* opts,
                                           void* stream);

/* vdx_search_batch_device without d_work, for callers that cannot allocate device memory (a
 * process whose HBM is handed out by an external pool manager, a real-time path that must not
 * call cudaMalloc, a plugin limited to the buffers its host passes in). No counterpart in the
 * reference, which has no device memory at all. Allocates nothing: the launch's work words live
 * in a 256-byte file-scope device array that every GPU loading this library holds until exit
 * (a launch needing more is rejected with VDX_ERR_LENGTH). The index must already have a
 * device copy for (opts->device, opts->precision): call vdx_index_upload first, which does
 * allocate. The first call on each device looks up the array's device address, so make it
 * before any stream capture; the address is kept for the life of the process, so resetting the
 * device afterwards (cudaDeviceReset) is not supported. All calls share the array and clear it
 * before their launch; calls whose kernels overlap on the GPU race on it, so serialize them.
 * Synchronous: returns after the batch finished, with the reference's error for a bad query
 * row. NULL query or result buffers (nq > 0), out_stride < k_uniform without d_k, and
 * opts->learned_stop (its network needs device memory the index allocates) are rejected with
 * VDX_ERR_INVALID_ARGUMENT before any launch. With d_k, a row's count never exceeds out_stride. */
VDX_API vdx_status vdx_search_batch_device_noalloc(const vdx_index* index, const float* d_queries,
                                                   uint64_t nq, uint64_t dim, const uint32_t* d_k,
                                                   const uint32_t* d_ef, uint32_t k_uniform,
                                                   uint32_t ef_uniform, uint32_t out_stride,
                                                   uint32_t* d_ids, float* d_dists,
                                                   uint32_t* d_counts,
                                                   const vdx_search_options* opts, void* stream);

/* --- Uneven batches through a captured CUDA graph (no counterpart in the reference) -------- */

typedef struct vdx_batcher vdx_batcher;
typedef struct vdx_plan_timing {
    uint32_t ef_class;          /* the class's largest effective ef */
    int32_t warps_per_block;
    uint32_t rows_per_round;
    uint32_t hash_slots;        /* visited-filter slots in shared memory (0 with a global table) */
    uint32_t result_capacity;
    float ms;
    uint32_t global_slots;      /* > 0: the visited filter is a global table of this many slots */
} vdx_plan_timing;

/* A batcher for batches of up to max_queries queries with per-query k <= max_k and
 * ef <= max_ef: device buffers, pinned staging and the search launches captured once into a
 * CUDA graph that every batch replays (the kernel reads the batch size, k and ef from device
 * memory). Queries are split into ef classes (effective ef <= 64, <= 256, <= 1024, ...), each
 * with its own launch plan, run as concurrent branches of the graph. Results equal
 * vdx_search_batch of each query with its own k and ef (BF16 / FP8: re-rank width 4 * k).
 * The batcher keeps the index's device copy as it was: adding to the index afterwards makes
 * every later run fail with VDX_ERR_INVALID_ARGUMENT. One batch at a time per batcher. */
VDX_API vdx_status vdx_batcher_create(const vdx_index* index, int32_t device, uint32_t precision,
                                      uint32_t max_queries, uint32_t max_k, uint32_t max_ef,
                                      vdx_batcher** out);
VDX_API void vdx_batcher_free(vdx_batcher* batcher);
/* One batch, synchronous: queries nq x dim (host), k_per_q, ef_per_q (host, nq each); results
 * ids / dists nq x max_k, counts nq. */
VDX_API vdx_status vdx_batcher_run(vdx_batcher* batcher, const float* queries, uint64_t nq,
                                   const uint32_t* k_per_q, const uint32_t* ef_per_q,
                                   uint32_t* ids, float* dists, uint32_t* counts);
/* vdx_batcher_run in two halves, so that several batchers keep several batches in flight:
 * submit copies the batch into the batcher's pinned staging and enqueues the copies and the graph
 * on its stream, without waiting (the caller's buffers may be reused at once); wait blocks until
 * that batch is done and writes ids / dists (nq x max_k) and counts. One batch in flight per
 * batcher: submit again before wait fails with VDX_ERR_INVALID_ARGUMENT. */
VDX_API vdx_status vdx_batcher_submit(vdx_batcher* batcher, const float* queries, uint64_t nq,
                                      const uint32_t* k_per_q, const uint32_t* ef_per_q);
VDX_API vdx_status vdx_batcher_wait(vdx_batcher* batcher, uint32_t* ids, float* dists,
                                    uint32_t* counts);
/* Times the candidate launch plans on a sample batch, keeps the fastest (and re-captures).
 * Up to `cap` timings are written to `timings`; *n_out receives how many plans were tried. */
VDX_API vdx_status vdx_batcher_autotune(vdx_batcher* batcher, const float* queries, uint64_t nq,
                                        const uint32_t* k_per_q, const uint32_t* ef_per_q,
                                        vdx_plan_timing* timings, uint64_t cap, uint64_t* n_out);

/* --- Learned early termination (no counterpart in the reference; its training and the
 * in-search network are this library's own) ------------------------------------------------ */

enum { VDX_STOP_PARAMS = 5057, VDX_STOP_FEATURES = 12 };

/* The model vdx_search_options.learned_stop uses: weights[5057] (W1 64x12, b1, W2 64x64, b2, W3,
 * b3), mean[12], inv_std[12], proj[4 x dim]. */
VDX_API vdx_status vdx_index_set_stop_model(vdx_index* index, const float* weights,
                                            const float* mean, const float* inv_std,
                                            const float* proj);
/* Training traces of the plain search at `ef` (see HnswIndex::trace_search): truth nq x
 * truth_k ids; features nq x max_points x 12; hits nq x max_points; points, final_hits nq. */
VDX_API vdx_status vdx_stop_trace(const vdx_index* index, const float* queries, uint64_t nq,
                                  uint64_t dim, const uint32_t* truth, uint64_t truth_k,
                                  uint64_t k, uint64_t ef, const float* proj, uint64_t max_points,
                                  float* features, uint8_t* hits, uint32_t* points,
                                  uint8_t* final_hits, int32_t device);
/* Trains the network on the GPU (own forward, backward and Adam kernels) on raw features
 * x[n][12] and labels y[n] in {0, 1}. Outputs weights[5057], mean[12], inv_std[12],
 * loss_per_epoch[epochs]. */
VDX_API vdx_status vdx_mlp_train(const float* x, const float* y, uint64_t n, uint32_t epochs,
                                 uint64_t batch, float lr, uint64_t seed, float* weights,
                                 float* mean, float* inv_std, float* loss_per_epoch);
/* One GPU forward + backward over standardized x: grad[5057] of the mean loss, and the loss. */
VDX_API vdx_status vdx_mlp_gradient(const float* x, const float* y, uint64_t n,
                                    const float* weights, float* grad, float* loss);
/* P(converged) for raw features x[n][12]. */
VDX_API vdx_status vdx_mlp_probabilities(const float* x, uint64_t n, const float* weights,
                                         const float* mean, const float* inv_std, float* prob);

/* --- BruteForceIndex ----------------------------------------------------------------------- */

/* BruteForceIndex(dim, metric): include/vecdex/brute_force.hpp:28 */
VDX_API vdx_status vdx_bf_create(uint64_t dim, uint32_t metric, vdx_bruteforce** out);
VDX_API void vdx_bf_free(vdx_bruteforce* index);
/* add(const Matrix<float>&): include/vecdex/brute_force.hpp:33 */
VDX_API vdx_status vdx_bf_add(vdx_bruteforce* index, const float* rows, uint64_t n,
                              uint64_t dim);
VDX_API uint64_t vdx_bf_size(const vdx_bruteforce* index);
/* search(query, k) for every row of `queries`: include/vecdex/brute_force.hpp:36
 * (src/brute_force.cpp:68-84), as one GPU batch. method: VDX_BF_EXACT or VDX_BF_TENSOR_CORE. */
VDX_API vdx_status vdx_bf_search_batch(const vdx_bruteforce* index, const float* queries,
                                       uint64_t nq, uint64_t dim, uint64_t k, uint32_t method,
                                       uint32_t* ids, float* dists, uint32_t* counts);

/* The device-buffer form of vdx_bf_search_batch, asynchronous on `stream`: d_queries nq x dim,
 * d_ids / d_dists nq x k, d_counts nq, d_work vdx_work_words() u32 ([0] error code, [1] first
 * failing row, [8] number of queries the tensor-core path recomputed exactly). */
VDX_API vdx_status vdx_bf_search_batch_device(const vdx_bruteforce* index, const float* d_queries,
                                              uint64_t nq, uint64_t dim, uint64_t k,
                                              uint32_t method, uint32_t* d_ids, float* d_dists,
                                              uint32_t* d_counts, uint32_t* d_work, void* stream);

/* No reference counterpart. For tests of the device-timeout path only: the limit, in
 * nanoseconds, of each pipeline wait of the tensor-core brute force's later launches in this
 * process (0 restores the default of 1 s). A limit shorter than a copy's latency makes the
 * launch give up (VDX_ERR_DEVICE_TIMEOUT) after draining its own copies and tensor-core work
 * with the full 1 s bound and freeing its tensor memory. */
VDX_API void vdx_testing_set_tc_wait_ns(uint64_t ns);

/* --- Host helpers (the distance kernels' order, the file checksum) -------------------------- */

/* kernels::active().l2_squared / inner_product: include/vecdex/kernels.hpp:31 */
VDX_API float vdx_host_l2(const float* a, const float* b, uint64_t dim);
VDX_API float vdx_host_ip(const float* a, const float* b, uint64_t dim);
/* XXH64 (the file checksum, docs/FORMAT.md "Checksum") */
VDX_API uint64_t vdx_xxh64(const void* data, uint64_t size, uint64_t seed);

#ifdef __cplusplus
}
#endif

#endif /* VDX_B200_H */
