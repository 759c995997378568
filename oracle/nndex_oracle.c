/*
 * nndex_oracle.c — CPU restatement of nndex's search path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker the CUDA backend is compared against and
 * the timed CPU baseline; it is never linked into, loaded by, or called from the product
 * library (nndex_b200/). Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use it.
 *
 * The reference (fblissjr/nndex) is Rust and cannot be compiled here (no cargo/rustc), so each
 * function below restates one reference function from its source, cited file:line. Third-party
 * arithmetic the reference calls but does not vendor is restated from its published behaviour:
 *   - simsimd 6.5.12 `f32::dot` (Cargo.toml:50): FP32 inputs, FP64 accumulation, the f64 result
 *     cast to f32 by the caller (src/cpu.rs:653-660, src/approx.rs:539-552, src/lib.rs:525-528).
 *   - ndarray 0.16.1 / matrixmultiply sgemm (Cargo.toml:45): FP32 multiply-accumulate; its
 *     blocking order is not reproducible, which only moves scores by a few FP32 ulps.
 * Parity is pinned by the golden vectors under tests/golden/ (reference tests and notebooks).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/nndex_cuda.h"

#define OR_API __attribute__((visibility("default")))

/* ============================================================================================
 * Arithmetic primitives
 * ========================================================================================== */

/* simsimd f32 dot: f64 accumulation of f32 products, returned as f64; callers cast to f32. */
static double simsimd_dot_f64(const float* a, const float* b, uint64_t n) {
    double s = 0.0;
    for (uint64_t i = 0; i < n; ++i) s += (double)a[i] * (double)b[i];
    return s;
}

/* src/cpu.rs:667-695 dot_unrolled_8: 8 FP32 accumulators, tail into s0, pairwise combine. */
OR_API float or_dot_unrolled_8(const float* lhs, const float* rhs, uint64_t len) {
    volatile float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint64_t idx = 0;
    while (idx + 8 <= len) {
        for (int j = 0; j < 8; ++j) {
            float p = lhs[idx + j] * rhs[idx + j];
            s[j] = s[j] + p;
        }
        idx += 8;
    }
    while (idx < len) {
        float p = lhs[idx] * rhs[idx];
        s[0] = s[0] + p;
        idx += 1;
    }
    return ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
}

/* src/cpu.rs:653-660 dot_product: simsimd when len >= 8, else dot_unrolled_8. */
OR_API float or_dot_product(const float* a, const float* b, uint64_t n) {
    if (n >= 8) return (float)simsimd_dot_f64(a, b, n);
    return or_dot_unrolled_8(a, b, n);
}

/* src/approx.rs:539-552 dot_small: simsimd when len >= 8, else a sequential FP32 sum. */
OR_API float or_dot_small(const float* a, const float* b, uint64_t n) {
    if (n >= 8) return (float)simsimd_dot_f64(a, b, n);
    volatile float sum = 0.0f;
    for (uint64_t i = 0; i < n; ++i) {
        float p = a[i] * b[i];
        sum = sum + p;
    }
    return sum;
}

/* Rust f32::total_cmp (used by src/topk.rs:28, 145, 197, 205): sign-magnitude → two's complement. */
static inline int32_t total_key(float f) {
    int32_t b;
    memcpy(&b, &f, 4);
    b ^= (int32_t)(((uint32_t)(b >> 31)) >> 1);
    return b;
}
static inline int total_cmp(float a, float b) {
    int32_t x = total_key(a), y = total_key(b);
    return (x > y) - (x < y);
}

/* ============================================================================================
 * Validation and normalisation (src/lib.rs:433-599)
 * ========================================================================================== */

/* src/lib.rs:433-442 validate_matrix_shape. */
OR_API int or_validate_matrix_shape(uint64_t n_values, uint64_t rows, uint64_t dims) {
    if (rows == 0 || dims == 0) return NNDEX_ERR_SHAPE_MISMATCH;
    unsigned __int128 p = (unsigned __int128)rows * dims;
    if (p > UINT64_MAX) p = UINT64_MAX; /* saturating_mul */
    if ((uint64_t)p != n_values) return NNDEX_ERR_SHAPE_MISMATCH;
    return NNDEX_OK;
}

/* src/lib.rs:445-450 ensure_finite. */
OR_API int or_ensure_finite(const float* v, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i)
        if (!isfinite(v[i])) return NNDEX_ERR_NON_FINITE;
    return NNDEX_OK;
}

/* src/lib.rs:519-553 normalize_row_into (cpu feature). */
static int normalize_row_into(const float* src, float* out, uint64_t dims, int prefer_simd) {
    float norm_sq;
    if (prefer_simd) {
        float sq = (float)simsimd_dot_f64(src, src, dims);
        if (!isfinite(sq)) return NNDEX_ERR_NON_FINITE;
        norm_sq = sq;
    } else {
        volatile float sq = 0.0f;
        for (uint64_t i = 0; i < dims; ++i) {
            if (!isfinite(src[i])) return NNDEX_ERR_NON_FINITE;
            float p = src[i] * src[i];
            sq = sq + p;
        }
        norm_sq = sq;
    }
    if (norm_sq <= FLT_EPSILON) return NNDEX_ERR_ZERO_NORM;
    volatile float root = sqrtf(norm_sq);
    volatile float inv = 1.0f / root;
    for (uint64_t i = 0; i < dims; ++i) out[i] = src[i] * inv;
    return NNDEX_OK;
}

/*
 * src/lib.rs:461-514 normalize_rows: rows are processed in order; the first failing row's error
 * is returned and its index stored in *bad_row. `out` is rows × padded, zero padded.
 * prefer_simd_norm = dims >= 16 (src/lib.rs:472-473).
 */
OR_API int or_normalize_rows(const float* v, uint64_t rows, uint64_t dims, uint64_t padded,
                             float* out, uint64_t* bad_row) {
    memset(out, 0, sizeof(float) * rows * padded);
    int prefer_simd = dims >= 16;
    for (uint64_t r = 0; r < rows; ++r) {
        int st = normalize_row_into(v + r * dims, out + r * padded, dims, prefer_simd);
        if (st != NNDEX_OK) {
            if (bad_row) *bad_row = r;
            return st;
        }
    }
    return NNDEX_OK;
}

/* src/lib.rs:558-575 normalize_vector: FP32 sequential norm with per-element finite check. */
OR_API int or_normalize_vector(const float* v, uint64_t dims, uint64_t padded, float* out) {
    volatile float norm_sq = 0.0f;
    for (uint64_t i = 0; i < dims; ++i) {
        if (!isfinite(v[i])) return NNDEX_ERR_NON_FINITE;
        float p = v[i] * v[i];
        norm_sq = norm_sq + p;
    }
    if (norm_sq <= FLT_EPSILON) return NNDEX_ERR_ZERO_NORM;
    volatile float root = sqrtf(norm_sq);
    volatile float inv = 1.0f / root;
    for (uint64_t i = 0; i < dims; ++i) out[i] = v[i] * inv;
    for (uint64_t i = dims; i < padded; ++i) out[i] = 0.0f;
    return NNDEX_OK;
}

/* src/lib.rs:578-588 pad_rows. */
OR_API void or_pad_rows(const float* v, uint64_t rows, uint64_t dims, uint64_t padded, float* out) {
    for (uint64_t r = 0; r < rows; ++r) {
        memcpy(out + r * padded, v + r * dims, sizeof(float) * dims);
        for (uint64_t i = dims; i < padded; ++i) out[r * padded + i] = 0.0f;
    }
}

/* src/lib.rs:192 padded_dims = dims.next_multiple_of(8). */
OR_API uint64_t or_padded_dims(uint64_t dims) { return (dims + 7) / 8 * 8; }

/* ============================================================================================
 * TopKAccumulator (src/topk.rs:44-152) — a faithful restatement of the bounded min-heap.
 * ========================================================================================== */

typedef struct {
    float sim;
    uint64_t idx;
} or_item;

/* HeapItem ordering (src/topk.rs:25-31): similarity by total_cmp, then index. */
static inline int item_lt(or_item a, or_item b) {
    int c = total_cmp(a.sim, b.sim);
    if (c != 0) return c < 0;
    return a.idx < b.idx;
}

typedef struct or_topk {
    uint64_t k;
    uint64_t len;
    or_item* heap; /* min-heap: heap[0] is the smallest (Reverse<HeapItem> max-heap top) */
    int has_best;
    or_item best;
    float min_threshold;
} or_topk;

/* src/topk.rs:55-62 new. */
OR_API or_topk* or_topk_new(uint64_t k) {
    or_topk* t = (or_topk*)calloc(1, sizeof(or_topk));
    t->k = k;
    t->heap = (or_item*)malloc(sizeof(or_item) * (k > 1 ? k + 1 : 1));
    t->min_threshold = -INFINITY;
    return t;
}
OR_API void or_topk_free(or_topk* t) {
    if (!t) return;
    free(t->heap);
    free(t);
}

static void heap_sift_down(or_item* h, uint64_t n, uint64_t i) {
    for (;;) {
        uint64_t l = 2 * i + 1, r = l + 1, m = i;
        if (l < n && item_lt(h[l], h[m])) m = l;
        if (r < n && item_lt(h[r], h[m])) m = r;
        if (m == i) return;
        or_item t = h[i];
        h[i] = h[m];
        h[m] = t;
        i = m;
    }
}
static void heap_sift_up(or_item* h, uint64_t i) {
    while (i > 0) {
        uint64_t p = (i - 1) / 2;
        if (!item_lt(h[i], h[p])) return;
        or_item t = h[i];
        h[i] = h[p];
        h[p] = t;
        i = p;
    }
}

/* src/topk.rs:80-105 push_slow. */
OR_API void or_topk_push_slow(or_topk* t, uint64_t index, float sim) {
    if (t->k == 1) {
        t->best.idx = index;
        t->best.sim = sim;
        t->has_best = 1;
        t->min_threshold = sim;
        return;
    }
    or_item it = {sim, index};
    if (t->len >= t->k) {
        t->heap[0] = it; /* peek_mut replaces the smallest, dropping it sifts down */
        heap_sift_down(t->heap, t->len, 0);
        t->min_threshold = t->heap[0].sim;
        return;
    }
    t->heap[t->len] = it;
    heap_sift_up(t->heap, t->len);
    t->len += 1;
    if (t->len == t->k) t->min_threshold = t->heap[0].sim;
}

/* src/topk.rs:70-75 push: fast reject `similarity <= min_threshold` (IEEE compare). */
OR_API void or_topk_push(or_topk* t, uint64_t index, float sim) {
    if (sim <= t->min_threshold) return;
    or_topk_push_slow(t, index, sim);
}

/* src/topk.rs:108-119 merge (consumes `o`; iterates o's heap storage order). */
OR_API void or_topk_merge(or_topk* t, or_topk* o) {
    if (t->k == 1) {
        if (o->has_best) or_topk_push(t, o->best.idx, o->best.sim);
    } else {
        for (uint64_t i = 0; i < o->len; ++i) or_topk_push(t, o->heap[i].idx, o->heap[i].sim);
    }
    or_topk_free(o);
}

static int neighbor_desc_cmp(const void* pa, const void* pb) {
    const or_item* a = (const or_item*)pa;
    const or_item* b = (const or_item*)pb;
    int c = total_cmp(b->sim, a->sim);
    if (c != 0) return c;
    return (a->idx > b->idx) - (a->idx < b->idx);
}

/* src/topk.rs:122-151 into_sorted_vec: similarity desc (total_cmp), index asc. Frees `t`. */
OR_API uint64_t or_topk_into_sorted(or_topk* t, uint64_t* idx, float* sim) {
    uint64_t n = 0;
    if (t->k == 1) {
        if (t->has_best) {
            idx[0] = t->best.idx;
            sim[0] = t->best.sim;
            n = 1;
        }
    } else {
        qsort(t->heap, t->len, sizeof(or_item), neighbor_desc_cmp);
        for (uint64_t i = 0; i < t->len; ++i) {
            idx[i] = t->heap[i].idx;
            sim[i] = t->heap[i].sim;
        }
        n = t->len;
    }
    or_topk_free(t);
    return n;
}

OR_API float or_topk_threshold(const or_topk* t) { return t->min_threshold; }

/* ---- canonical selection: the k best by (similarity desc, index asc) ------------------ */

/* "a is better than b" under the canonical order. */
static inline int canon_better(float sa, uint64_t ia, float sb, uint64_t ib) {
    int c = total_cmp(sa, sb);
    if (c != 0) return c > 0;
    return ia < ib;
}

typedef struct {
    uint64_t k, len;
    or_item* h; /* min-heap under "worse first": h[0] is the worst kept item */
} canon_heap;

static inline int canon_worse(or_item a, or_item b) { return canon_better(b.sim, b.idx, a.sim, a.idx); }

static void canon_sift_down(or_item* h, uint64_t n, uint64_t i) {
    for (;;) {
        uint64_t l = 2 * i + 1, r = l + 1, m = i;
        if (l < n && canon_worse(h[l], h[m])) m = l;
        if (r < n && canon_worse(h[r], h[m])) m = r;
        if (m == i) return;
        or_item t = h[i];
        h[i] = h[m];
        h[m] = t;
        i = m;
    }
}
static void canon_push(canon_heap* c, float sim, uint64_t idx) {
    if (c->k == 0) return;
    or_item it = {sim, idx};
    if (c->len < c->k) {
        uint64_t i = c->len++;
        c->h[i] = it;
        while (i > 0) {
            uint64_t p = (i - 1) / 2;
            if (!canon_worse(c->h[i], c->h[p])) break;
            or_item t = c->h[i];
            c->h[i] = c->h[p];
            c->h[p] = t;
            i = p;
        }
        return;
    }
    if (!canon_better(sim, idx, c->h[0].sim, c->h[0].idx)) return;
    c->h[0] = it;
    canon_sift_down(c->h, c->len, 0);
}
static uint64_t canon_finish(canon_heap* c, uint64_t* idx, float* sim) {
    qsort(c->h, c->len, sizeof(or_item), neighbor_desc_cmp);
    for (uint64_t i = 0; i < c->len; ++i) {
        idx[i] = c->h[i].idx;
        sim[i] = c->h[i].sim;
    }
    return c->len;
}

/*
 * src/topk.rs:169-210 topk_from_scores. len > 131072: streaming through push_slow with the
 * hoisted threshold; else quickselect + sort, i.e. the canonical top-k.
 */
OR_API uint64_t or_topk_from_scores(const float* scores, uint64_t n, uint64_t k, uint64_t offset,
                                    uint64_t* idx, float* sim) {
    uint64_t capped = k < n ? k : n;
    if (capped == 0) return 0;
    if (n > 131072) {
        or_topk* acc = or_topk_new(capped);
        float threshold = acc->min_threshold;
        for (uint64_t i = 0; i < n; ++i) {
            if (scores[i] > threshold) {
                or_topk_push_slow(acc, i + offset, scores[i]);
                threshold = acc->min_threshold;
            }
        }
        return or_topk_into_sorted(acc, idx, sim);
    }
    canon_heap c = {capped, 0, (or_item*)malloc(sizeof(or_item) * capped)};
    for (uint64_t i = 0; i < n; ++i) canon_push(&c, scores[i], i + offset);
    uint64_t m = canon_finish(&c, idx, sim);
    free(c.h);
    return m;
}

/* ============================================================================================
 * Exact search
 * ========================================================================================== */

/*
 * Canonical exact top-k of every query over `base` (rows × dp, normalised and padded), scored
 * with the reference's dot_product (src/cpu.rs:653-660: simsimd, FP64 accumulate → f32) and
 * selected by (similarity desc, index asc) — the order `topk_from_scores` and `into_sorted_vec`
 * return (src/topk.rs:143-148, 204-208). Outputs are nq × k (k already capped at rows).
 * Parallel over row chunks per query; per-chunk canonical selections merge exactly.
 */
OR_API void or_search_exact(const float* base, uint64_t rows, uint64_t dp, const float* queries,
                            uint64_t nq, uint64_t k, uint64_t* idx_out, float* sim_out) {
    const uint64_t chunk = 8192;
    uint64_t nchunks = (rows + chunk - 1) / chunk;
    or_item* part = (or_item*)malloc(sizeof(or_item) * nchunks * (k ? k : 1));
    uint64_t* plen = (uint64_t*)malloc(sizeof(uint64_t) * nchunks);
    for (uint64_t q = 0; q < nq; ++q) {
        const float* qv = queries + q * dp;
#pragma omp parallel for schedule(dynamic, 1)
        for (uint64_t c = 0; c < nchunks; ++c) {
            canon_heap h = {k, 0, part + c * k};
            uint64_t r0 = c * chunk, r1 = r0 + chunk < rows ? r0 + chunk : rows;
            for (uint64_t r = r0; r < r1; ++r) canon_push(&h, or_dot_product(base + r * dp, qv, dp), r);
            plen[c] = h.len;
        }
        canon_heap all = {k, 0, (or_item*)malloc(sizeof(or_item) * (k ? k : 1))};
        for (uint64_t c = 0; c < nchunks; ++c)
            for (uint64_t i = 0; i < plen[c]; ++i) canon_push(&all, part[c * k + i].sim, part[c * k + i].idx);
        canon_finish(&all, idx_out + q * k, sim_out + q * k);
        free(all.h);
    }
    free(part);
    free(plen);
}

/* FP64 ground truth: exact dot products of the stored FP32 rows and queries in double. */
OR_API void or_scores_f64(const float* base, uint64_t rows, uint64_t dp, const float* query,
                          double* out) {
#pragma omp parallel for schedule(static)
    for (uint64_t r = 0; r < rows; ++r) {
        const float* x = base + r * dp;
        double s = 0.0;
        for (uint64_t d = 0; d < dp; ++d) s += (double)x[d] * (double)query[d];
        out[r] = s;
    }
}

/* FP64 top-(k) by (score desc, index asc) for one query, plus the (k+1)-th score (or -inf). */
OR_API void or_search_f64(const float* base, uint64_t rows, uint64_t dp, const float* query,
                          uint64_t k, uint64_t* idx_out, double* score_out, double* next_score) {
    double* s = (double*)malloc(sizeof(double) * rows);
    or_scores_f64(base, rows, dp, query, s);
    uint64_t kk = k + 1 < rows ? k + 1 : rows;
    /* simple selection of kk best with a small sorted insertion buffer */
    uint64_t* bi = (uint64_t*)malloc(sizeof(uint64_t) * (kk ? kk : 1));
    double* bs = (double*)malloc(sizeof(double) * (kk ? kk : 1));
    uint64_t n = 0;
    for (uint64_t r = 0; r < rows; ++r) {
        double v = s[r];
        if (n == kk && !(v > bs[n - 1])) continue;
        uint64_t pos = n < kk ? n : kk - 1;
        while (pos > 0 && v > bs[pos - 1]) {
            bs[pos] = bs[pos - 1];
            bi[pos] = bi[pos - 1];
            --pos;
        }
        bs[pos] = v;
        bi[pos] = r;
        if (n < kk) ++n;
    }
    uint64_t m = k < n ? k : n;
    for (uint64_t i = 0; i < m; ++i) {
        idx_out[i] = bi[i];
        score_out[i] = bs[i];
    }
    *next_score = n > k ? bs[k] : -INFINITY;
    free(bi);
    free(bs);
    free(s);
}

/* ============================================================================================
 * IVF (src/approx.rs) — parameterised restatement; defaults are the reference policy.
 * ========================================================================================== */

/* src/approx.rs:339-350 isqrt (Newton). */
OR_API uint64_t or_isqrt(uint64_t n) {
    if (n == 0) return 0;
    uint64_t x = n, y = (x + 1) / 2;
    while (y < x) {
        x = y;
        y = (x + n / x) / 2;
    }
    return x;
}

/* src/approx.rs:305-311 choose_nlist. */
OR_API uint64_t or_choose_nlist(uint64_t rows) {
    if (rows < 256) return 1;
    uint64_t s = or_isqrt(rows);
    return s < 16 ? 16 : (s > 512 ? 512 : s);
}

/* src/approx.rs:318-336 choose_nprobe. */
OR_API uint64_t or_choose_nprobe(uint64_t nlist, uint64_t k, uint64_t rows) {
    uint64_t pct = k >= 50 ? 8 : (k >= 20 ? 6 : 4);
    uint64_t nprobe = (nlist * pct + 99) / 100;
    if (nprobe < 1) nprobe = 1;
    uint64_t nl = nlist ? nlist : 1;
    uint64_t avg = rows / nl;
    if (avg < 1) avg = 1;
    unsigned __int128 mc = (unsigned __int128)k * 40;
    uint64_t min_cand = mc > UINT64_MAX ? UINT64_MAX : (uint64_t)mc;
    uint64_t min_nprobe = (min_cand + avg - 1) / avg;
    if (min_nprobe < 1) min_nprobe = 1;
    if (nprobe < min_nprobe) nprobe = min_nprobe;
    if (nprobe < 1) nprobe = 1;
    if (nprobe > nlist) nprobe = nlist;
    return nprobe;
}

/* src/approx.rs:409-429 pick_medoid_row. */
OR_API uint64_t or_pick_medoid_row(const float* m, uint64_t rows, uint64_t dims) {
    double* mean = (double*)calloc(dims, sizeof(double));
    for (uint64_t r = 0; r < rows; ++r)
        for (uint64_t d = 0; d < dims; ++d) mean[d] += (double)m[r * dims + d];
    double inv_rows = 1.0 / (double)rows;
    float* mf = (float*)malloc(sizeof(float) * dims);
    for (uint64_t d = 0; d < dims; ++d) mf[d] = (float)(mean[d] * inv_rows);
    float* dots = (float*)malloc(sizeof(float) * rows);
#pragma omp parallel for schedule(static)
    for (uint64_t r = 0; r < rows; ++r) dots[r] = or_dot_small(m + r * dims, mf, dims);
    uint64_t best = 0;
    float best_dot = -INFINITY;
    for (uint64_t r = 0; r < rows; ++r)
        if (dots[r] > best_dot) {
            best_dot = dots[r];
            best = r;
        }
    free(mean);
    free(mf);
    free(dots);
    return best;
}

/*
 * src/approx.rs:357-406 kmeans_plusplus_init. The LCG start state is rows*2654435761+dims
 * (wrapping) unless `has_seed`, in which case it is `seed`. `chosen_rows` (nlist) receives the
 * row picked for each centroid (the medoid first; a duplicate of the previous pick when the
 * total distance is zero).
 */
OR_API void or_kmeans_plusplus_init(const float* m, uint64_t rows, uint64_t dims, uint64_t nlist,
                                    int has_seed, uint64_t seed, float* centroids,
                                    uint64_t* chosen_rows) {
    uint64_t rng = has_seed ? seed : rows * 2654435761ull + dims;
    uint64_t first = or_pick_medoid_row(m, rows, dims);
    memcpy(centroids, m + first * dims, sizeof(float) * dims);
    if (chosen_rows) chosen_rows[0] = first;
    uint64_t last_row = first;
    float* min_d = (float*)malloc(sizeof(float) * rows);
    for (uint64_t r = 0; r < rows; ++r) min_d[r] = FLT_MAX;
    for (uint64_t c = 1; c < nlist; ++c) {
        const float* last = centroids + (c - 1) * dims;
#pragma omp parallel for schedule(static)
        for (uint64_t r = 0; r < rows; ++r) {
            float dot = or_dot_small(m + r * dims, last, dims);
            float dist = 1.0f - dot;
            if (!(dist >= 0.0f)) dist = 0.0f; /* f32::max(0.0): negative or NaN → 0 */
            if (dist < min_d[r]) min_d[r] = dist;
        }
        double total = 0.0;
        for (uint64_t r = 0; r < rows; ++r) total += (double)min_d[r];
        if (total <= 0.0) {
            memcpy(centroids + c * dims, last, sizeof(float) * dims);
            if (chosen_rows) chosen_rows[c] = last_row;
            continue;
        }
        rng = rng * 6364136223846793005ull + 1ull;
        double threshold = ((double)rng / (double)UINT64_MAX) * total;
        double cum = 0.0;
        uint64_t chosen = rows - 1;
        for (uint64_t r = 0; r < rows; ++r) {
            cum += (double)min_d[r];
            if (cum >= threshold) {
                chosen = r;
                break;
            }
        }
        memcpy(centroids + c * dims, m + chosen * dims, sizeof(float) * dims);
        if (chosen_rows) chosen_rows[c] = chosen;
        last_row = chosen;
    }
    free(min_d);
}

/*
 * The assignment step of src/approx.rs:446-493 for `n` rows of `m` (their indices in `row_ids`):
 * the strict `>` argmax of dot_small over the centroids, so the lowest centroid index wins ties.
 */
OR_API void or_kmeans_assign_rows(const float* m, uint64_t dims, const uint64_t* row_ids, uint64_t n,
                                  const float* centroids, uint64_t nlist, uint32_t* assign) {
#pragma omp parallel for schedule(dynamic, 256)
    for (uint64_t i = 0; i < n; ++i) {
        const float* row = m + row_ids[i] * dims;
        uint32_t best_c = 0;
        float best_s = -INFINITY;
        for (uint64_t c = 0; c < nlist; ++c) {
            float s = or_dot_small(row, centroids + c * dims, dims);
            if (s > best_s) {
                best_s = s;
                best_c = (uint32_t)c;
            }
        }
        assign[i] = best_c;
    }
}

/*
 * The update step of src/approx.rs:495-531 from an assignment: FP64 sums in row order, mean,
 * renormalise with the 1e-30 guard, empty cluster → zero centroid; written into `centroids`.
 */
OR_API void or_kmeans_update(const float* m, uint64_t rows, uint64_t dims, uint64_t nlist,
                             const uint32_t* assign, float* centroids) {
    double* sums = (double*)calloc(nlist * dims, sizeof(double));
    uint64_t* sizes = (uint64_t*)calloc(nlist, sizeof(uint64_t));
    for (uint64_t r = 0; r < rows; ++r) {
        uint32_t c = assign[r];
        sizes[c] += 1;
        const float* row = m + r * dims;
        double* s = sums + (uint64_t)c * dims;
        for (uint64_t d = 0; d < dims; ++d) s[d] += (double)row[d];
    }
    for (uint64_t c = 0; c < nlist; ++c) {
        float* out = centroids + c * dims;
        if (sizes[c] == 0) {
            for (uint64_t d = 0; d < dims; ++d) out[d] = 0.0f;
            continue;
        }
        double inv_count = 1.0 / (double)sizes[c];
        const double* s = sums + c * dims;
        double norm_sq = 0.0;
        for (uint64_t d = 0; d < dims; ++d) {
            double scaled = s[d] * inv_count;
            norm_sq += scaled * scaled;
        }
        double inv_norm = norm_sq > 1e-30 ? 1.0 / sqrt(norm_sq) : 1.0;
        for (uint64_t d = 0; d < dims; ++d) out[d] = (float)(s[d] * inv_count * inv_norm);
    }
    free(sums);
    free(sizes);
}

/*
 * src/approx.rs:434-535 spherical_kmeans for `iters` iterations: assignment by strict `>`
 * argmax of dot_small (lowest centroid index wins ties), FP64 sums in row order, mean,
 * renormalise with the 1e-30 guard, empty cluster → zero centroid. `assign` receives the
 * assignments of the last iteration (made against the centroids before its update).
 */
OR_API void or_spherical_kmeans(const float* m, uint64_t rows, uint64_t dims, uint64_t nlist,
                                uint64_t iters, float* centroids, uint32_t* assign) {
    uint64_t* all = (uint64_t*)malloc(sizeof(uint64_t) * rows);
    for (uint64_t r = 0; r < rows; ++r) all[r] = r;
    for (uint64_t it = 0; it < iters; ++it) {
        or_kmeans_assign_rows(m, dims, all, rows, centroids, nlist, assign);
        or_kmeans_update(m, rows, dims, nlist, assign, centroids);
    }
    free(all);
}

typedef struct or_ivf {
    uint64_t rows, dims, nlist;
    float* centroids;          /* nlist × dims                                     */
    float* reordered;          /* rows × dims, cluster-contiguous                  */
    uint64_t* original;        /* rows: position → original row                    */
    uint64_t* offsets;         /* nlist + 1                                        */
    uint32_t* assign;          /* rows: final assignment per original row          */
    uint64_t* init_rows;       /* nlist: rows picked by k-means++                  */
} or_ivf;

/*
 * src/approx.rs:46-100 ApproxIndex::build. `nlist` 0 = choose_nlist(rows); `iters` 0 = 12.
 * rows < 256 or nlist < 2 → the single-list index (src/approx.rs:49-59).
 */
OR_API or_ivf* or_ivf_build(const float* m, uint64_t rows, uint64_t dims, uint64_t nlist,
                            uint64_t iters, int has_seed, uint64_t seed) {
    or_ivf* ix = (or_ivf*)calloc(1, sizeof(or_ivf));
    ix->rows = rows;
    ix->dims = dims;
    if (nlist == 0) nlist = or_choose_nlist(rows);
    if (iters == 0) iters = 12;
    ix->reordered = (float*)malloc(sizeof(float) * rows * dims);
    ix->original = (uint64_t*)malloc(sizeof(uint64_t) * rows);
    ix->assign = (uint32_t*)calloc(rows, sizeof(uint32_t));
    if (rows < 256 || nlist < 2) {
        ix->nlist = 1;
        memcpy(ix->reordered, m, sizeof(float) * rows * dims);
        for (uint64_t r = 0; r < rows; ++r) ix->original[r] = r;
        ix->offsets = (uint64_t*)malloc(sizeof(uint64_t) * 2);
        ix->offsets[0] = 0;
        ix->offsets[1] = rows;
        return ix;
    }
    ix->nlist = nlist;
    ix->centroids = (float*)malloc(sizeof(float) * nlist * dims);
    ix->init_rows = (uint64_t*)malloc(sizeof(uint64_t) * nlist);
    or_kmeans_plusplus_init(m, rows, dims, nlist, has_seed, seed, ix->centroids, ix->init_rows);
    or_spherical_kmeans(m, rows, dims, nlist, iters, ix->centroids, ix->assign);
    uint64_t* counts = (uint64_t*)calloc(nlist, sizeof(uint64_t));
    for (uint64_t r = 0; r < rows; ++r) counts[ix->assign[r]] += 1;
    ix->offsets = (uint64_t*)malloc(sizeof(uint64_t) * (nlist + 1));
    ix->offsets[0] = 0;
    for (uint64_t c = 0; c < nlist; ++c) ix->offsets[c + 1] = ix->offsets[c] + counts[c];
    uint64_t* wp = (uint64_t*)malloc(sizeof(uint64_t) * nlist);
    memcpy(wp, ix->offsets, sizeof(uint64_t) * nlist);
    for (uint64_t r = 0; r < rows; ++r) {
        uint64_t dst = wp[ix->assign[r]]++;
        ix->original[dst] = r;
        memcpy(ix->reordered + dst * dims, m + r * dims, sizeof(float) * dims);
    }
    free(wp);
    free(counts);
    return ix;
}

/*
 * An index over a given layout (centroids, offsets, original_indices, as ApproxIndex holds them,
 * src/approx.rs:11-25): the reordered rows are gathered from `m`. Lets the CPU baseline time the
 * reference's search on an index built elsewhere (the build itself is timed separately).
 */
OR_API or_ivf* or_ivf_from_layout(const float* m, uint64_t rows, uint64_t dims, uint64_t nlist,
                                  const float* centroids, const uint64_t* offsets,
                                  const uint64_t* original) {
    or_ivf* ix = (or_ivf*)calloc(1, sizeof(or_ivf));
    ix->rows = rows;
    ix->dims = dims;
    ix->nlist = nlist;
    ix->centroids = (float*)malloc(sizeof(float) * nlist * dims);
    memcpy(ix->centroids, centroids, sizeof(float) * nlist * dims);
    ix->offsets = (uint64_t*)malloc(sizeof(uint64_t) * (nlist + 1));
    memcpy(ix->offsets, offsets, sizeof(uint64_t) * (nlist + 1));
    ix->original = (uint64_t*)malloc(sizeof(uint64_t) * rows);
    memcpy(ix->original, original, sizeof(uint64_t) * rows);
    ix->reordered = (float*)malloc(sizeof(float) * rows * dims);
#pragma omp parallel for schedule(static)
    for (uint64_t p = 0; p < rows; ++p)
        memcpy(ix->reordered + p * dims, m + original[p] * dims, sizeof(float) * dims);
    ix->assign = (uint32_t*)calloc(rows, sizeof(uint32_t));
    return ix;
}

OR_API void or_ivf_free(or_ivf* ix) {
    if (!ix) return;
    free(ix->centroids);
    free(ix->reordered);
    free(ix->original);
    free(ix->offsets);
    free(ix->assign);
    free(ix->init_rows);
    free(ix);
}

OR_API uint64_t or_ivf_nlist(const or_ivf* ix) { return ix->nlist; }
OR_API const float* or_ivf_centroids(const or_ivf* ix) { return ix->centroids; }
OR_API const uint64_t* or_ivf_offsets(const or_ivf* ix) { return ix->offsets; }
OR_API const uint64_t* or_ivf_original(const or_ivf* ix) { return ix->original; }
OR_API const uint32_t* or_ivf_assign(const or_ivf* ix) { return ix->assign; }
OR_API const uint64_t* or_ivf_init_rows(const or_ivf* ix) { return ix->init_rows; }
/* src/approx.rs:35-37 provides_speedup. */
OR_API int or_ivf_provides_speedup(const or_ivf* ix) { return ix->rows >= 256 && ix->nlist >= 4; }

/*
 * src/approx.rs:159-215 candidate_clusters: centroid scores, then the nprobe best clusters.
 * The reference's select_nth_unstable_by compares scores only, so ties among centroid scores are
 * unordered there; here they go to the lower cluster index. Centroid scores use dot_small
 * (FP64-accumulated) — the reference uses ndarray sgemv when nlist >= 16 and dims >= 16, whose
 * FP32 rounding differs by a few ulps. Writes nprobe cluster ids into `clusters` (probe order =
 * score desc, index asc) and returns nprobe.
 */
OR_API uint64_t or_ivf_probe(const or_ivf* ix, const float* query, uint64_t nprobe,
                             uint64_t* clusters, float* cscores) {
    if (ix->nlist <= 1) {
        clusters[0] = 0;
        if (cscores) cscores[0] = 0.0f;
        return 1;
    }
    if (nprobe > ix->nlist) nprobe = ix->nlist;
    canon_heap h = {nprobe, 0, (or_item*)malloc(sizeof(or_item) * nprobe)};
    for (uint64_t c = 0; c < ix->nlist; ++c)
        canon_push(&h, or_dot_small(ix->centroids + c * ix->dims, query, ix->dims), c);
    float* sims = (float*)malloc(sizeof(float) * nprobe);
    uint64_t n = canon_finish(&h, clusters, sims);
    if (cscores) memcpy(cscores, sims, sizeof(float) * n);
    free(sims);
    free(h.h);
    return n;
}

/*
 * src/cpu.rs:425-453 search_approx: exact FP32 rerank of the probed clusters, selected by the
 * canonical order. `nprobe` 0 = choose_nprobe(nlist, k, rows). Returns the result count (< k
 * when the probed clusters hold fewer rows).
 */
OR_API uint64_t or_ivf_search(const or_ivf* ix, const float* query, uint64_t k, uint64_t nprobe,
                              uint64_t* idx_out, float* sim_out) {
    if (nprobe == 0) nprobe = or_choose_nprobe(ix->nlist, k, ix->rows);
    uint64_t np = ix->nlist <= 1 ? 1 : (nprobe < ix->nlist ? nprobe : ix->nlist);
    uint64_t* cl = (uint64_t*)malloc(sizeof(uint64_t) * np);
    np = or_ivf_probe(ix, query, np, cl, NULL);
    canon_heap h = {k, 0, (or_item*)malloc(sizeof(or_item) * (k ? k : 1))};
    for (uint64_t i = 0; i < np; ++i) {
        uint64_t s = ix->offsets[cl[i]], e = ix->offsets[cl[i] + 1];
        for (uint64_t p = s; p < e; ++p)
            canon_push(&h, or_dot_product(ix->reordered + p * ix->dims, query, ix->dims), ix->original[p]);
    }
    uint64_t n = canon_finish(&h, idx_out, sim_out);
    free(h.h);
    free(cl);
    return n;
}

/* Batch form of or_ivf_search (src/cpu.rs:456-502), parallel over queries. */
OR_API void or_ivf_search_batch(const or_ivf* ix, const float* queries, uint64_t nq, uint64_t k,
                                uint64_t nprobe, uint64_t* idx_out, float* sim_out,
                                uint64_t* counts) {
#pragma omp parallel for schedule(dynamic, 1)
    for (uint64_t q = 0; q < nq; ++q)
        counts[q] = or_ivf_search(ix, queries + q * ix->dims, k, nprobe, idx_out + q * k, sim_out + q * k);
}

/* ============================================================================================
 * Timed CPU baseline: the reference's exact CPU strategies, multithreaded on the host cores.
 * ========================================================================================== */

OR_API int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
OR_API void or_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* FP32 dot with 16 independent lanes (vectorises to AVX2/AVX-512 FMA; the simsimd role). */
__attribute__((optimize("fp-contract=fast"))) static inline float fast_dot(const float* a, const float* b, uint64_t n) {
    float acc[16] = {0};
    uint64_t i = 0;
    for (; i + 16 <= n; i += 16)
        for (int j = 0; j < 16; ++j) acc[j] += a[i + j] * b[i + j];
    for (; i < n; ++i) acc[0] += a[i] * b[i];
    float s = 0.0f;
    for (int j = 0; j < 16; ++j) s += acc[j];
    return s;
}

/*
 * Single query: src/cpu.rs:594-639 ParallelChunked / ParallelFold — row chunks scored with
 * dot products into per-thread TopKAccumulators (src/topk.rs:70-105), merged (src/topk.rs:108).
 */
OR_API uint64_t or_bench_search_single(const float* base, uint64_t rows, uint64_t dp,
                                       const float* q, uint64_t k, uint64_t* idx, float* sim) {
    int nt = or_num_threads();
    or_topk** accs = (or_topk**)malloc(sizeof(or_topk*) * nt);
    for (int t = 0; t < nt; ++t) accs[t] = or_topk_new(k);
#pragma omp parallel
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        or_topk* acc = accs[t];
#pragma omp for schedule(static, 64)
        for (uint64_t r = 0; r < rows; ++r) or_topk_push(acc, r, fast_dot(base + r * dp, q, dp));
    }
    for (int t = 1; t < nt; ++t) or_topk_merge(accs[0], accs[t]);
    uint64_t n = or_topk_into_sorted(accs[0], idx, sim);
    free(accs);
    return n;
}

/*
 * Score blocks for the batch baseline: S[q][r] = dot(query q, row r) for a block of rows × queries,
 * by a register-blocked FP32 micro-kernel (4 rows × 4 queries of vector accumulators along D, the
 * matrixmultiply role in the reference's sgemm), chosen at run time: AVX-512 (16 lanes, 16 zmm
 * accumulators) where the host has it, else AVX2 (8 lanes, 2 rows × 4 queries). Timing only: the
 * summation order is the kernel's, not the reference's.
 */
#if defined(__x86_64__)
#include <immintrin.h>

__attribute__((target("avx512f"))) static void micro_4x4_avx512(const float* r0, const float* r1, const float* r2,
                                                                const float* r3, const float* const* q,
                                                                uint64_t dp, float out[4][4]) {
    __m512 acc[4][4];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) acc[i][j] = _mm512_setzero_ps();
    const float* rr[4] = {r0, r1, r2, r3};
    uint64_t d = 0;
    for (; d + 16 <= dp; d += 16) {
        __m512 x[4], y[4];
        for (int i = 0; i < 4; ++i) x[i] = _mm512_loadu_ps(rr[i] + d);
        for (int j = 0; j < 4; ++j) y[j] = _mm512_loadu_ps(q[j] + d);
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) acc[i][j] = _mm512_fmadd_ps(x[i], y[j], acc[i][j]);
    }
    if (d < dp) {  /* padded dims are a multiple of 8: one masked half step */
        const __mmask16 m = (__mmask16)((1u << (dp - d)) - 1u);
        __m512 x[4], y[4];
        for (int i = 0; i < 4; ++i) x[i] = _mm512_maskz_loadu_ps(m, rr[i] + d);
        for (int j = 0; j < 4; ++j) y[j] = _mm512_maskz_loadu_ps(m, q[j] + d);
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) acc[i][j] = _mm512_fmadd_ps(x[i], y[j], acc[i][j]);
    }
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) out[i][j] = _mm512_reduce_add_ps(acc[i][j]);
}

__attribute__((target("avx2,fma"))) static void micro_2x4_avx2(const float* r0, const float* r1,
                                                               const float* const* q, uint64_t dp, float out[2][4]) {
    __m256 acc[2][4];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 4; ++j) acc[i][j] = _mm256_setzero_ps();
    for (uint64_t d = 0; d + 8 <= dp; d += 8) {
        const __m256 x0 = _mm256_loadu_ps(r0 + d), x1 = _mm256_loadu_ps(r1 + d);
        for (int j = 0; j < 4; ++j) {
            const __m256 y = _mm256_loadu_ps(q[j] + d);
            acc[0][j] = _mm256_fmadd_ps(x0, y, acc[0][j]);
            acc[1][j] = _mm256_fmadd_ps(x1, y, acc[1][j]);
        }
    }
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 4; ++j) {
            __m128 v = _mm_add_ps(_mm256_castps256_ps128(acc[i][j]), _mm256_extractf128_ps(acc[i][j], 1));
            v = _mm_add_ps(v, _mm_movehl_ps(v, v));
            v = _mm_add_ss(v, _mm_shuffle_ps(v, v, 1));
            out[i][j] = _mm_cvtss_f32(v);
        }
}

static int host_has_avx512(void) {
    static int v = -1;
    if (v < 0) v = __builtin_cpu_supports("avx512f") ? 1 : 0;
    return v;
}
#endif

/* Scores of rows [rb, re) of `base` against queries [qb, qe) into scores[q * ld + (r - rofs)]. */
static void score_block(const float* base, uint64_t dp, uint64_t rb, uint64_t re, uint64_t rofs, const float* qs,
                        uint64_t qb, uint64_t qe, float* scores, uint64_t ld) {
    uint64_t q = qb;
#if defined(__x86_64__)
    const int wide = host_has_avx512();
    for (; q + 4 <= qe; q += 4) {
        const float* qp[4] = {qs + q * dp, qs + (q + 1) * dp, qs + (q + 2) * dp, qs + (q + 3) * dp};
        uint64_t r = rb;
        if (wide) {
            for (; r + 4 <= re; r += 4) {
                float o[4][4];
                micro_4x4_avx512(base + r * dp, base + (r + 1) * dp, base + (r + 2) * dp, base + (r + 3) * dp, qp, dp, o);
                for (int i = 0; i < 4; ++i)
                    for (int j = 0; j < 4; ++j) scores[(q + j) * ld + (r + i - rofs)] = o[i][j];
            }
        } else {
            for (; r + 2 <= re; r += 2) {
                float o[2][4];
                micro_2x4_avx2(base + r * dp, base + (r + 1) * dp, qp, dp, o);
                for (int i = 0; i < 2; ++i)
                    for (int j = 0; j < 4; ++j) scores[(q + j) * ld + (r + i - rofs)] = o[i][j];
            }
        }
        for (; r < re; ++r)
            for (int j = 0; j < 4; ++j) scores[(q + j) * ld + (r - rofs)] = fast_dot(base + r * dp, qp[j], dp);
    }
#endif
    for (; q < qe; ++q)
        for (uint64_t r = rb; r < re; ++r) scores[q * ld + (r - rofs)] = fast_dot(base + r * dp, qs + q * dp, dp);
}

/*
 * Batch: src/cpu.rs:256-284 Gemm (score matrix in blocks, then topk_from_scores per query) or
 * src/cpu.rs:291-341 GemmChunked (64 MB base chunks streamed into per-query accumulators), as
 * src/profiles.rs:151-185 picks for (rows, dims, nq). Each thread scores a block of 64 rows against
 * every query (the block stays in its core's cache while the queries pass over it, so the base is
 * read from memory once per batch) with the register-blocked micro-kernel of score_block.
 */
OR_API void or_bench_search_batch(const float* base, uint64_t rows, uint64_t dp, const float* qs,
                                  uint64_t nq, uint64_t k, uint64_t* idx, float* sim) {
    uint64_t score_bytes = nq * rows * 4;
    int chunked = score_bytes > 128ull * 1024 * 1024;
    uint64_t chunk_rows = chunked ? ((64ull * 1024 * 1024) / (dp * 4)) : rows;
    if (chunk_rows < 64) chunk_rows = 64;
    if (chunk_rows > rows) chunk_rows = rows;
    float* scores = (float*)malloc(sizeof(float) * nq * chunk_rows);
    or_topk** accs = (or_topk**)malloc(sizeof(or_topk*) * nq);
    for (uint64_t q = 0; q < nq; ++q) accs[q] = or_topk_new(k);
    for (uint64_t r0 = 0; r0 < rows; r0 += chunk_rows) {
        uint64_t nr = rows - r0 < chunk_rows ? rows - r0 : chunk_rows;
        const uint64_t RB = 64, QB = 64;
#pragma omp parallel for schedule(dynamic, 1)
        for (uint64_t rb = 0; rb < nr; rb += RB) {
            uint64_t re = rb + RB < nr ? rb + RB : nr;
            for (uint64_t qb = 0; qb < nq; qb += QB) {
                uint64_t qe = qb + QB < nq ? qb + QB : nq;
                score_block(base, dp, r0 + rb, r0 + re, r0, qs, qb, qe, scores, chunk_rows);
            }
        }
        if (!chunked) {
#pragma omp parallel for schedule(dynamic, 1)
            for (uint64_t q = 0; q < nq; ++q) {
                or_topk_free(accs[q]);
                accs[q] = NULL;
                or_topk_from_scores(scores + q * chunk_rows, nr, k, 0, idx + q * k, sim + q * k);
            }
        } else {
#pragma omp parallel for schedule(dynamic, 1)
            for (uint64_t q = 0; q < nq; ++q) {
                or_topk* acc = accs[q];
                float thr = acc->min_threshold;
                const float* s = scores + q * chunk_rows;
                for (uint64_t i = 0; i < nr; ++i)
                    if (s[i] > thr) {
                        or_topk_push_slow(acc, r0 + i, s[i]);
                        thr = acc->min_threshold;
                    }
            }
        }
    }
    if (chunked)
        for (uint64_t q = 0; q < nq; ++q) or_topk_into_sorted(accs[q], idx + q * k, sim + q * k);
    free(accs);
    free(scores);
}
