/*
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE: the oracle.
 *
 * A plain-C CPU restatement of the vecdex batched query path, used only by tests/, smoke() and
 * bench.py's CPU-baseline leg as the checker. It is pinned against the unmodified reference
 * (oracle/_ref/libvecdex_ref.so, built from the reference's own sources) and against the
 * reference's published golden fingerprints (tests/hnsw_parallel_test.cpp:146-169); see
 * tests/test_oracle.py. Every function names the reference code it restates
 * (paths relative to the reference project).
 *
 * Besides results, the traversal counts the events the reference cannot report (expansions,
 * distance evaluations, link-list and vector bytes read), which cross-check the GPU kernels'
 * device counters and size the roofline's algorithmic bytes.
 *
 * Compiled with -ffp-contract=off: every multiply-add below is explicit (fmaf or a separate
 * product and sum), exactly as the reference's AVX2 kernels round.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------ */
/* Distance kernels: src/kernels_avx2.cpp:17-80 (the kernel set the reference picks on any    */
/* x86-64 host with AVX2+FMA, src/kernels.cpp:160-176).                                       */
/*                                                                                            */
/* Accumulator lane (j, l), j = 0..3, l = 0..7, runs an FMA chain over elements 32t + 8j + l;  */
/* then 8-wide steps into accumulator 0; then (acc0 + acc1) + (acc2 + acc3) lane-wise; then    */
/* the fixed horizontal tree of horizontal_sum (:17-22): ((v0+v4)+(v2+v6)) + ((v1+v5)+(v3+v7)); */
/* then a sequential tail of dim % 8 elements. How the tail rounds is up to the compiler that */
/* built the reference: GCC 13.3 -O3 (the reference's Release flags) contracts `sum += x * y`  */
/* into one FMA (in C++ it applies -ffp-contract=off only to ISO C), except that it first     */
/* SLP-vectorizes the products (and, for L2, the differences) of the first four tail elements  */
/* when the tail has at least four: those four are rounded as products, then added in order.  */
/* Measured bitwise against oracle/_ref on every dim 0..100 and the common embedding sizes     */
/* (tests/test_oracle.py). Tail modes: 0 = that GCC 13.3 build (default), 1 = every tail term */
/* fused, 2 = none fused.                                                                      */
/* ------------------------------------------------------------------------------------------ */

static int g_tail_mode = 0;

void vo_set_tail_mode(int mode) { g_tail_mode = mode; }

static float avx2_order(const float* a, const float* b, uint64_t dim, int l2) {
    float acc[4][8];
    memset(acc, 0, sizeof acc);
    uint64_t i = 0;
    for (; dim - i >= 32; i += 32) {
        for (int j = 0; j < 4; ++j) {
            for (int l = 0; l < 8; ++l) {
                const uint64_t e = i + 8 * (uint64_t)j + (uint64_t)l;
                if (l2) {
                    const float d = a[e] - b[e];
                    acc[j][l] = fmaf(d, d, acc[j][l]);
                } else {
                    acc[j][l] = fmaf(a[e], b[e], acc[j][l]);
                }
            }
        }
    }
    for (; dim - i >= 8; i += 8) {
        for (int l = 0; l < 8; ++l) {
            const uint64_t e = i + (uint64_t)l;
            if (l2) {
                const float d = a[e] - b[e];
                acc[0][l] = fmaf(d, d, acc[0][l]);
            } else {
                acc[0][l] = fmaf(a[e], b[e], acc[0][l]);
            }
        }
    }
    float v[8];
    for (int l = 0; l < 8; ++l) {
        v[l] = (acc[0][l] + acc[1][l]) + (acc[2][l] + acc[3][l]);
    }
    const float h0 = v[0] + v[4], h1 = v[1] + v[5], h2 = v[2] + v[6], h3 = v[3] + v[7];
    float sum = (h0 + h2) + (h1 + h3);
    const uint64_t tail_start = i;
    const uint64_t tail = dim - i;
    for (; i < dim; ++i) {
        const float x = l2 ? a[i] - b[i] : a[i];
        const float y = l2 ? x : b[i];
        int fused = g_tail_mode != 2;
        if (g_tail_mode == 0 && tail >= 4 && i - tail_start < 4) {
            fused = 0;
        }
        if (fused) {
            sum = fmaf(x, y, sum);
        } else {
            const float p = x * y;
            sum = sum + p;
        }
    }
    return sum;
}

float vo_l2(const float* a, const float* b, uint64_t dim) { return avx2_order(a, b, dim, 1); }
float vo_ip(const float* a, const float* b, uint64_t dim) { return avx2_order(a, b, dim, 0); }

/* Metric codes as in the file format (docs/FORMAT.md "Header"): 0 L2, 1 IP, 2 cosine.
 * IP and cosine rank by 1 - <a, b> (src/hnsw.cpp:202-205, src/distance.cpp:10-30). */
static float metric_distance(int metric, const float* a, const float* b, uint64_t dim) {
    if (metric == 0) {
        return vo_l2(a, b, dim);
    }
    return 1.0f - vo_ip(a, b, dim);
}

/* src/vector_ops.cpp:14-34 and :78-86: n = sqrt(<v, v>) with the active kernel, then x /= n. */
void vo_normalize(float* v, uint64_t dim) {
    const float n = sqrtf(vo_ip(v, v, dim));
    for (uint64_t i = 0; i < dim; ++i) {
        v[i] /= n;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Neighbor order: include/vecdex/neighbor.hpp:23-25. Smaller distance first, ties by id.     */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    float d;
    uint32_t id;
} vo_nb;

static int closer(vo_nb a, vo_nb b) { return a.d < b.d || (a.d == b.d && a.id < b.id); }

/* Binary heaps with the std::push_heap / pop_heap contract: `less(a, b)` orders the heap so that
 * the greatest element under `less` sits at index 0. Which element is "greatest" is all that
 * matters for the search; the tie-free total order makes every heap discipline agree. */
typedef int (*vo_less)(vo_nb, vo_nb);

static int farther(vo_nb a, vo_nb b) { return closer(b, a); }

static void heap_push(vo_nb* h, size_t* n, vo_nb x, vo_less less) {
    size_t i = (*n)++;
    h[i] = x;
    while (i > 0) {
        const size_t p = (i - 1) / 2;
        if (!less(h[p], h[i])) {
            break;
        }
        const vo_nb t = h[p];
        h[p] = h[i];
        h[i] = t;
        i = p;
    }
}

static vo_nb heap_pop(vo_nb* h, size_t* n, vo_less less) {
    const vo_nb top = h[0];
    h[0] = h[--(*n)];
    size_t i = 0;
    for (;;) {
        const size_t l = 2 * i + 1, r = l + 1;
        size_t m = i;
        if (l < *n && less(h[m], h[l])) {
            m = l;
        }
        if (r < *n && less(h[m], h[r])) {
            m = r;
        }
        if (m == i) {
            break;
        }
        const vo_nb t = h[m];
        h[m] = h[i];
        h[i] = t;
        i = m;
    }
    return top;
}

static int cmp_closer(const void* pa, const void* pb) {
    const vo_nb a = *(const vo_nb*)pa, b = *(const vo_nb*)pb;
    return closer(a, b) ? -1 : (closer(b, a) ? 1 : 0);
}

/* ------------------------------------------------------------------------------------------ */
/* The index file, docs/FORMAT.md (reader: src/hnsw_io.cpp:409-467). This restatement only    */
/* reads valid files; the product's reader is the one that treats files as hostile.           */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    uint64_t dim, M, n, max_level, entry, upper_blocks;
    int metric;
    uint8_t* levels;
    uint32_t* layer0;    /* n blocks of 1 + 2M: [count, ids...] */
    uint32_t* upper;     /* U blocks of 1 + M */
    uint64_t* upper_at;  /* per node: index of its layer-1 block in `upper` */
    float* vectors;      /* n x dim */
} vo_index;

void vo_index_free(vo_index* ix) {
    if (!ix) {
        return;
    }
    free(ix->levels);
    free(ix->layer0);
    free(ix->upper);
    free(ix->upper_at);
    free(ix->vectors);
    free(ix);
}

vo_index* vo_index_load(const char* path) {
    FILE* f = fopen(path, "rb");
    if (!f) {
        return NULL;
    }
    unsigned char h[80];
    vo_index* ix = (vo_index*)calloc(1, sizeof *ix);
    if (fread(h, 1, 80, f) != 80 || memcmp(h, "\x89VDXHNSW", 8) != 0) {
        fclose(f);
        free(ix);
        return NULL;
    }
    uint32_t metric;
    memcpy(&metric, h + 12, 4);
    ix->metric = (int)metric;
    memcpy(&ix->dim, h + 16, 8);
    memcpy(&ix->M, h + 24, 8);
    memcpy(&ix->n, h + 48, 8);
    memcpy(&ix->max_level, h + 56, 8);
    memcpy(&ix->entry, h + 64, 8);
    memcpy(&ix->upper_blocks, h + 72, 8);
    const uint64_t n = ix->n, b0 = 1 + 2 * ix->M, b1 = 1 + ix->M;
    ix->levels = (uint8_t*)malloc(n ? n : 1);
    ix->layer0 = (uint32_t*)malloc((n * b0 != 0 ? n * b0 : 1) * 4);
    ix->upper = (uint32_t*)malloc((ix->upper_blocks * b1 != 0 ? ix->upper_blocks * b1 : 1) * 4);
    ix->upper_at = (uint64_t*)malloc((n ? n : 1) * 8);
    ix->vectors = (float*)malloc((n * ix->dim != 0 ? n * ix->dim : 1) * 4);
    int ok = fread(ix->levels, 1, n, f) == n && fread(ix->layer0, 4, n * b0, f) == n * b0 &&
             fread(ix->upper, 4, ix->upper_blocks * b1, f) == ix->upper_blocks * b1 &&
             fread(ix->vectors, 4, n * ix->dim, f) == n * ix->dim;
    fclose(f);
    if (!ok) {
        vo_index_free(ix);
        return NULL;
    }
    uint64_t at = 0;
    for (uint64_t i = 0; i < n; ++i) {
        ix->upper_at[i] = at;
        at += ix->levels[i];
    }
    return ix;
}

uint64_t vo_index_size(const vo_index* ix) { return ix->n; }
uint64_t vo_index_dim(const vo_index* ix) { return ix->dim; }
int vo_index_metric(const vo_index* ix) { return ix->metric; }

/* src/hnsw.cpp:151-165: [count, ids...] of `node` on `layer`. */
static const uint32_t* links(const vo_index* ix, uint64_t node, uint64_t layer) {
    if (layer == 0) {
        return ix->layer0 + node * (1 + 2 * ix->M);
    }
    return ix->upper + (ix->upper_at[node] + layer - 1) * (1 + ix->M);
}

static const float* vec(const vo_index* ix, uint64_t id) { return ix->vectors + id * ix->dim; }

/* ------------------------------------------------------------------------------------------ */
/* Traversal copies of the stored vectors (no reference counterpart: the reference searches     */
/* FP32 only). What the GPU traversal reads, as the FP32 values it computes with:               */
/*   BF16: every element rounded to bfloat16, round to nearest, ties to even;                   */
/*   FP8:  one FP32 scale per row, s = max|x| / 448 (1 when the row is zero), every element     */
/*         x / s rounded to E4M3 (1-4-3, bias 7, max finite 448, subnormal quantum 2^-9),       */
/*         round to nearest, ties to even, saturating at +-448, then read back as s * e4m3.     */
/* Distances then follow the reference's kernel order on these values (FP32 accumulation).     */
/* ------------------------------------------------------------------------------------------ */

float vo_bf16_round(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    u += 0x7FFFu + ((u >> 16) & 1u); /* half of the dropped range, plus one on an odd kept lsb */
    u &= 0xFFFF0000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

float vo_e4m3_round(float v) {
    const float a = fabsf(v);
    float r;
    if (a >= 448.0F) {
        r = 448.0F;
    } else {
        int e2;
        (void)frexpf(a, &e2);                         /* a = f * 2^e2, f in [0.5, 1) */
        const int e = a >= 0x1p-6F ? e2 - 1 : -6;     /* binade exponent; subnormals share 2^-6 */
        const float quantum = ldexpf(1.0F, e - 3);    /* 3 mantissa bits */
        r = rintf(a / quantum) * quantum;             /* exact scaling; rintf rounds half to even */
    }
    return copysignf(r, v); /* E4M3 keeps the sign of zero too */
}

void vo_quantize_rows(int precision, const float* in, uint64_t n, uint64_t dim, float* out) {
    for (uint64_t i = 0; i < n; ++i) {
        const float* x = in + i * dim;
        float* y = out + i * dim;
        if (precision == 1) {
            for (uint64_t e = 0; e < dim; ++e) {
                y[e] = vo_bf16_round(x[e]);
            }
        } else if (precision == 2) {
            float m = 0.0F;
            for (uint64_t e = 0; e < dim; ++e) {
                m = fmaxf(m, fabsf(x[e]));
            }
            const float s = m > 0.0F ? m / 448.0F : 1.0F;
            for (uint64_t e = 0; e < dim; ++e) {
                y[e] = s * vo_e4m3_round(x[e] / s);
            }
        } else {
            memcpy(y, x, dim * 4);
        }
    }
}

/* Replaces a loaded index's vectors by their traversal copy (precision 1 BF16, 2 FP8). */
void vo_index_quantize(vo_index* ix, int precision) {
    vo_quantize_rows(precision, ix->vectors, ix->n, ix->dim, ix->vectors);
}

/* ------------------------------------------------------------------------------------------ */
/* Search: src/hnsw.cpp:416-522.                                                              */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    uint64_t expansions;      /* layer-0 nodes whose links were read */
    uint64_t dist_layer0;     /* distance evaluations on layer 0 */
    uint64_t dist_upper;      /* distance evaluations on layers >= 1 (including the entry) */
    uint64_t link_bytes;      /* link blocks read: 4 * (1 + count) each */
    uint64_t upper_hops;      /* upper-layer link lists read */
} vo_stats;

/* greedy_closest, src/hnsw.cpp:416-431: scan links in order, move on a strictly smaller
 * distance (distance only, not id), repeat until a whole pass makes no move. */
static vo_nb greedy_closest(const vo_index* ix, const float* q, vo_nb entry, uint64_t layer,
                            vo_stats* st) {
    for (int moved = 1; moved;) {
        moved = 0;
        const uint32_t* block = links(ix, entry.id, layer);
        const uint32_t count = block[0];
        st->upper_hops += 1;
        st->link_bytes += 4ull * (1 + count);
        for (uint32_t i = 0; i < count; ++i) {
            const uint32_t id = block[1 + i];
            const float d = metric_distance(ix->metric, q, vec(ix, id), ix->dim);
            st->dist_upper += 1;
            if (d < entry.d) {
                entry.d = d;
                entry.id = id;
                moved = 1;
            }
        }
    }
    return entry;
}

typedef struct {
    uint32_t* marks; /* src/search_scratch.hpp:21-47: epoch-stamped visited list */
    uint32_t epoch;
    uint64_t cap;
    vo_nb* cand;
    vo_nb* res;
    uint32_t* fresh;
} vo_scratch;

static void scratch_reset(vo_scratch* s, uint64_t n, uint64_t ef, uint64_t max_links) {
    if (s->cap < n) {
        free(s->marks);
        s->marks = (uint32_t*)calloc(n ? n : 1, 4);
        s->cap = n;
        s->epoch = 0;
    }
    if (++s->epoch == 0) {
        memset(s->marks, 0, s->cap * 4);
        s->epoch = 1;
    }
    (void)ef;
    (void)max_links;
}

/* search_layer, src/hnsw.cpp:438-482, on layer 0: candidate min-heap (front = closest),
 * result max-heap (front = worst), stop when full and the worst result is closer than the
 * closest candidate; every unvisited neighbor is scored, and admitted while results are short
 * of ef or it beats the worst result. Returns |results|; results are left sorted (closest
 * first), as sort_heap leaves them in search_unchecked (:519). */
static size_t search_layer0(const vo_index* ix, const float* q, vo_nb entry, uint64_t ef,
                            vo_scratch* s, vo_stats* st) {
    const uint64_t cap0 = 2 * ix->M;
    /* The heaps never hold more than ef + 1 results, or more candidates than scored nodes. */
    size_t nc = 0, nr = 0;
    s->marks[entry.id] = s->epoch;
    heap_push(s->cand, &nc, entry, farther);
    heap_push(s->res, &nr, entry, closer);
    while (nc > 0) {
        const vo_nb cur = heap_pop(s->cand, &nc, farther);
        if (nr >= ef && closer(s->res[0], cur)) {
            break;
        }
        const uint32_t* block = links(ix, cur.id, 0);
        const uint32_t count = block[0];
        st->expansions += 1;
        st->link_bytes += 4ull * (1 + count);
        size_t nf = 0;
        for (uint32_t i = 0; i < count && i < cap0; ++i) {
            const uint32_t id = block[1 + i];
            if (s->marks[id] != s->epoch) {
                s->marks[id] = s->epoch;
                s->fresh[nf++] = id;
            }
        }
        for (size_t i = 0; i < nf; ++i) {
            const vo_nb next = {metric_distance(ix->metric, q, vec(ix, s->fresh[i]), ix->dim),
                                s->fresh[i]};
            st->dist_layer0 += 1;
            if (nr < ef || closer(next, s->res[0])) {
                heap_push(s->cand, &nc, next, farther);
                heap_push(s->res, &nr, next, closer);
                if (nr > ef) {
                    (void)heap_pop(s->res, &nr, closer);
                }
            }
        }
    }
    qsort(s->res, nr, sizeof(vo_nb), cmp_closer);
    return nr;
}

/* search_unchecked, src/hnsw.cpp:504-522 (the caller has validated the query, :484-488). */
static uint32_t search_one(const vo_index* ix, const float* query, uint64_t k, uint64_t ef,
                           vo_scratch* s, vo_stats* st, uint32_t* ids, float* dists) {
    for (uint64_t i = 0; i < k; ++i) {
        ids[i] = 0xFFFFFFFFu;
        dists[i] = INFINITY;
    }
    if (ix->n == 0) {
        return 0;
    }
    float* qn = NULL;
    const float* q = query;
    if (ix->metric == 2) {
        qn = (float*)malloc(ix->dim * 4);
        memcpy(qn, query, ix->dim * 4);
        vo_normalize(qn, ix->dim);
        q = qn;
    }
    const uint64_t efk = ef > k ? ef : k;
    scratch_reset(s, ix->n, efk, 2 * ix->M);
    vo_nb entry = {metric_distance(ix->metric, q, vec(ix, ix->entry), ix->dim),
                   (uint32_t)ix->entry};
    st->dist_upper += 1;
    for (uint64_t layer = ix->max_level; layer > 0; --layer) {
        entry = greedy_closest(ix, q, entry, layer, st);
    }
    const size_t nr = search_layer0(ix, q, entry, efk, s, st);
    const uint64_t out = nr < k ? nr : k;
    for (uint64_t i = 0; i < out; ++i) {
        ids[i] = s->res[i].id;
        dists[i] = s->res[i].d;
    }
    free(qn);
    return (uint32_t)out;
}

/* Sequential search over a batch (search_batch's per-row contract, include/vecdex/hnsw.hpp:95-99).
 * `stats` (optional) receives one vo_stats per query. Queries must be valid. */
void vo_search_batch(const vo_index* ix, const float* queries, uint64_t nq, uint64_t k,
                     uint64_t ef, uint32_t* ids, float* dists, uint32_t* counts,
                     uint64_t* stats) {
    vo_scratch s;
    memset(&s, 0, sizeof s);
    const uint64_t efk = ef > k ? ef : k;
    /* Candidates: at most one push per scored node; results: at most ef + 1. */
    const uint64_t room = ix->n + 2;
    s.cand = (vo_nb*)malloc(room * sizeof(vo_nb));
    s.res = (vo_nb*)malloc((efk + 2 > room ? efk + 2 : room) * sizeof(vo_nb));
    s.fresh = (uint32_t*)malloc((2 * ix->M + 1) * 4);
    for (uint64_t q = 0; q < nq; ++q) {
        vo_stats st;
        memset(&st, 0, sizeof st);
        counts[q] = search_one(ix, queries + q * ix->dim, k, ef, &s, &st, ids + q * k,
                               dists + q * k);
        if (stats) {
            uint64_t* o = stats + q * 5;
            o[0] = st.expansions;
            o[1] = st.dist_layer0;
            o[2] = st.dist_upper;
            o[3] = st.link_bytes;
            o[4] = st.upper_hops;
        }
    }
    free(s.marks);
    free(s.cand);
    free(s.res);
    free(s.fresh);
}

/* ------------------------------------------------------------------------------------------ */
/* Brute force: src/brute_force.cpp:19-37 (select_top_k) and :68-84 (search). Rows are stored  */
/* normalized under cosine (:58-66); `base` here is already as the index stores it.           */
/* ------------------------------------------------------------------------------------------ */

void vo_bruteforce_batch(const float* base, uint64_t n, uint64_t dim, int metric,
                         const float* queries, uint64_t nq, uint64_t k, uint32_t* ids,
                         float* dists, uint32_t* counts) {
    const uint64_t keep = k < n ? k : n;
    vo_nb* heap = (vo_nb*)malloc((keep + 1) * sizeof(vo_nb));
    float* qn = (float*)malloc(dim * 4);
    for (uint64_t q = 0; q < nq; ++q) {
        memcpy(qn, queries + q * dim, dim * 4);
        if (metric == 2) {
            vo_normalize(qn, dim);
        }
        size_t nh = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const vo_nb c = {metric_distance(metric, qn, base + i * dim, dim), (uint32_t)i};
            if (nh < keep) {
                heap_push(heap, &nh, c, closer);
            } else if (keep > 0 && closer(c, heap[0])) {
                (void)heap_pop(heap, &nh, closer);
                heap_push(heap, &nh, c, closer);
            }
        }
        qsort(heap, nh, sizeof(vo_nb), cmp_closer);
        for (uint64_t i = 0; i < k; ++i) {
            ids[q * k + i] = i < nh ? heap[i].id : 0xFFFFFFFFu;
            dists[q * k + i] = i < nh ? heap[i].d : INFINITY;
        }
        counts[q] = (uint32_t)nh;
    }
    free(heap);
    free(qn);
}

/* The FNV-1a results fingerprint of tests/hnsw_parallel_test.cpp:91-105 (ids and distance bits
 * of every result, no per-list length), over rows of `counts[q]` results padded to k. */
uint64_t vo_fingerprint(const uint32_t* ids, const float* dists, const uint32_t* counts,
                        uint64_t nq, uint64_t k) {
    uint64_t hash = 14695981039346656037ull;
    for (uint64_t q = 0; q < nq; ++q) {
        for (uint64_t i = 0; i < counts[q]; ++i) {
            uint32_t words[2];
            words[0] = ids[q * k + i];
            memcpy(&words[1], &dists[q * k + i], 4);
            for (int w = 0; w < 2; ++w) {
                for (unsigned shift = 0; shift < 32; shift += 8) {
                    hash = (hash ^ ((words[w] >> shift) & 0xFFu)) * 1099511628211ull;
                }
            }
        }
    }
    return hash;
}

/* ------------------------------------------------------------------------------------------ */
/* Fixtures. integer_matrix of tests/hnsw_parallel_test.cpp:37-48: std::mt19937(seed) (the     */
/* 32-bit Mersenne Twister with its standard init_genrand seeding, fully specified by the C++  */
/* standard), each value the top 8 bits of one draw minus 128.                                */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    uint32_t mt[624];
    int idx;
} vo_mt19937;

static void mt_seed(vo_mt19937* g, uint32_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 624; ++i) {
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    }
    g->idx = 624;
}

static uint32_t mt_next(vo_mt19937* g) {
    if (g->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            const uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

void vo_integer_matrix(uint64_t rows, uint64_t dim, uint32_t seed, float* out) {
    vo_mt19937 g;
    mt_seed(&g, seed);
    for (uint64_t i = 0; i < rows * dim; ++i) {
        out[i] = (float)((int)(mt_next(&g) >> 24) - 128);
    }
}
