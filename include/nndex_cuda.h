/*
 * nndex_cuda.h — C ABI of the B200 (sm_100a) backend for nndex's cosine top-k search path.
 *
 * This is the seam a `BackendImpl::Cuda(Arc<CudaIndex>)` arm binds to in nndex
 * (src/lib.rs:147-154 `enum BackendImpl`, src/lib.rs:246-269 `match options.backend`).
 * Every entry point takes plain pointers and sizes; no C++ or CUDA runtime types cross it
 * (streams are passed as `void*`). No exception or abort crosses the ABI: every call returns
 * an `int` status (0 = OK) and leaves a thread-local message behind `nndex_cuda_last_error()`.
 *
 * Status codes map 1:1 onto nndex's `NNdexError` (src/lib.rs:107-145); the CUDA-specific
 * failures map onto one new variant `NNdexError::Cuda(String)`, the analogue of
 * `NNdexError::Gpu(#[from] GpuError)` (src/lib.rs:141-144).
 *
 * Results follow nndex's `Neighbor` contract (src/topk.rs:6-11): index as `uint64_t`,
 * similarity as `float`, sorted by similarity descending and, for equal similarity,
 * by index ascending (src/topk.rs:143-148, src/topk.rs:268-281).
 */
#ifndef NNDEX_CUDA_H
#define NNDEX_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define NNDEX_API __attribute__((visibility("default")))
#else
#define NNDEX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (NNdexError, src/lib.rs:107-145) ------------------------------------ */
#define NNDEX_OK                   0
#define NNDEX_ERR_SHAPE_MISMATCH   1  /* NNdexError::ShapeMismatch{rows,dims,values}      */
#define NNDEX_ERR_QUERY_DIMS       2  /* NNdexError::QueryDimensionalityMismatch           */
#define NNDEX_ERR_INVALID_TOPK     3  /* NNdexError::InvalidTopK                           */
#define NNDEX_ERR_NON_FINITE       4  /* NNdexError::NonFiniteInput                        */
#define NNDEX_ERR_ZERO_NORM        5  /* NNdexError::ZeroNorm                              */
#define NNDEX_ERR_CUDA             6  /* NNdexError::Cuda: a CUDA runtime/driver failure   */
#define NNDEX_ERR_OUT_OF_MEMORY    7  /* NNdexError::Cuda: device allocation failed        */
#define NNDEX_ERR_TIMEOUT          8  /* NNdexError::Cuda: a bounded device wait ran out   */
#define NNDEX_ERR_ADMISSION        9  /* NNdexError::Cuda: serving admission refused       */
#define NNDEX_ERR_INVALID_ARGUMENT 10 /* NNdexError::Cuda: bad handle / pointer / option    */
#define NNDEX_ERR_DEVICE_INDEX     11 /* GpuError::DeviceIndexOutOfRange (src/gpu.rs:46-52) */
#define NNDEX_ERR_UNSUPPORTED      12 /* NNdexError::Cuda: request outside compiled limits  */
#define NNDEX_PENDING              13 /* serving: the request has not finished (not an error) */

/* ---- construction flags (IndexOptions, src/lib.rs:64-77) ------------------------------- */
#define NNDEX_FLAG_NORMALIZED 0x1u /* IndexOptions::normalized: rows/queries already unit  */
#define NNDEX_FLAG_APPROX     0x2u /* IndexOptions::approx: IVF prefilter + exact rerank    */
#define NNDEX_FLAG_BF16       0x4u /* keep a BF16 scoring copy (tensor-core scan + rerank)  */
#define NNDEX_FLAG_FP8        0x8u /* keep an FP8-E4M3 scoring copy with per-row scales     */

/* ---- precision of the exact scan ------------------------------------------------------ */
#define NNDEX_PRECISION_AUTO 0u /* autotuner: FP32 at small batches, low precision + rerank */
#define NNDEX_PRECISION_FP32 1u /* plain FP32 scan (CUDA cores)                               */
#define NNDEX_PRECISION_BF16 2u /* BF16 tensor-core scan + exact FP32 rerank                  */
#define NNDEX_PRECISION_FP8  3u /* FP8-E4M3 tensor-core scan + exact FP32 rerank              */

/* Hard limits of the compiled kernels. */
#define NNDEX_MAX_DIMS 16384u       /* padded dimensionality                                 */
#define NNDEX_MAX_ROWS 4294967295ull /* row indices travel as 32-bit inside the kernels      */

typedef struct nndex_cuda_index nndex_cuda_index;

/*
 * Options that nndex's IndexOptions does not carry. All-zero means "reference policy":
 *   nlist   = clamp(isqrt(rows), 16, 512)        (src/approx.rs:305-311 choose_nlist)
 *   nprobe  = choose_nprobe(nlist, k, rows)      (src/approx.rs:318-336)
 *   iters   = 12                                 (src/approx.rs:28 KMEANS_MAX_ITERS)
 *   seed    = rows * 2654435761 + padded_dims    (src/approx.rs:359-361)
 * `device` is IndexOptions::gpu_device_index (src/lib.rs:76); -1 selects device 0.
 */
typedef struct nndex_cuda_opts {
    int32_t  device;          /* CUDA ordinal, -1 = default (0)                              */
    uint32_t precision;       /* NNDEX_PRECISION_*                                           */
    uint32_t nlist;           /* 0 = reference policy                                        */
    uint32_t nprobe;          /* 0 = reference policy (per-search, depends on k)             */
    uint32_t kmeans_iters;    /* 0 = 12                                                      */
    uint32_t has_seed;        /* 1 = use `seed` as the k-means++ LCG start state             */
    uint64_t seed;
    uint32_t rerank_width;    /* k' for low-precision scans; 0 = autotuned                    */
    uint32_t reserved[7];
} nndex_cuda_opts;

/* Device description (GpuDeviceInfo, src/gpu.rs:974-987), CUDA flavoured. */
typedef struct nndex_cuda_devinfo {
    uint64_t index;            /* CUDA ordinal                                              */
    char     name[256];        /* cudaDeviceProp::name                                      */
    char     driver[64];       /* "NVIDIA"                                                  */
    char     driver_info[64];  /* driver and runtime versions                              */
    char     backend[32];      /* "Cuda"                                                    */
    char     device_type[32];  /* "DiscreteGpu"                                             */
    uint32_t sm_count;
    uint32_t cc_major, cc_minor;
    uint64_t hbm_bytes;
    uint64_t l2_bytes;
} nndex_cuda_devinfo;

/* Search-side statistics of the last call on this index (per index, not thread-local). */
typedef struct nndex_cuda_search_stats {
    uint32_t path;             /* 1 = FP32 scan, 2 = BF16 scan+rerank, 3 = FP8 scan+rerank,
                                  4 = IVF probe + rerank, 5 = IVF list scan on the tensor
                                  cores + rerank, 6 = TF32 candidate scan + rerank
                                  (9-16 queries of a batch)                                    */
    uint32_t kernel_launches;  /* kernels this library launched for the call                */
    uint32_t rerank_width;     /* k' of a low-precision scan's first pass (0 otherwise)     */
    uint32_t certified;        /* 1 = every query certified after the first pass            */
    uint32_t second_pass_queries;   /* queries that took the threshold-collection pass     */
    uint32_t nprobe;           /* IVF lists probed per query                                */
    uint64_t rows_scanned;     /* base rows scored (sum over queries for IVF)               */
    double   device_ms;        /* CUDA-event time of the device part of the call            */
    uint32_t fp32_fallback_queries; /* queries re-run on the FP32 scan (pass-2 overflow, or
                                       an uncertified query of path 6)                       */
    uint32_t pass1_tile_stride;     /* first pass scanned every n-th 256-row tile (1 = all) */
    uint64_t ivf_rows_streamed;     /* IVF: rows read by the list scan (a list once per query group) */
    uint64_t ivf_rows_union;        /* IVF: rows in the union of the probed lists               */
    uint32_t scan_qb;               /* FP32 scan: queries per CTA of its last launch            */
    uint32_t scan_wide;             /* FP32 scan: 0 = 4-row × 8-query warps, 7 / 8 / 11 / 16 =
                                       consumer warps of 16 rows × all queries (wide consumer)  */
    uint32_t graph;                 /* host-buffer search: 0 = direct launches, 1 = captured as a
                                       CUDA graph by this call, 2 = a cached graph replayed      */
    uint32_t score_errors;          /* 1 = the call measured every result's score error        */
    double   max_score_error;       /* largest |score − FP64 score| over the call's results     */
    double   mean_score_error;      /* their mean (both 0 unless score_errors)                  */
    uint32_t tuned;                 /* plan of the call's last batch: 0 = by the rules, 1 = the
                                       autotuner timed the candidates on it, 2 = from the tuner's
                                       cache                                                     */
    uint32_t tune_candidates;       /* plans the autotuner compared for that shape (0 = none)    */
    uint64_t pass2_rows;            /* tensor-core paths: rows the second pass collected (summed
                                       over its queries) and re-scored in FP32                  */
    uint32_t pass2_query_blocks;    /* paths 2/3: 128-query blocks per CTA of the second pass
                                       (2 = two blocks against 128-row base tiles; 3 = one block
                                       per CTA of a CTA pair sharing 256-row tiles; 0 = no pass) */
    uint32_t reserved0;
} nndex_cuda_search_stats;

/* IVF build statistics (approximate mode; zero when the index has no IVF). */
typedef struct nndex_cuda_ivf_stats {
    uint64_t nlist;            /* clusters                                                   */
    uint64_t iters;            /* k-means iterations run                                     */
    uint64_t max_list;         /* rows of the largest cluster                                */
    double   build_ms;         /* whole build, device time                                   */
    double   seed_ms;          /* medoid + k-means++ seeding                                 */
    double   kmeans_ms;        /* the k-means iterations                                     */
    double   layout_ms;        /* list layout: reordered rows, row map, offsets              */
    uint64_t seed_exact_rows;  /* rows whose seeding distance was computed exactly           */
    uint64_t ambiguous_rows;   /* assignments re-scored against every centroid (all iters)   */
    uint64_t candidate_rows;   /* assignments decided exactly among <= 3 candidates (all iters) */
    uint64_t reserved[3];
} nndex_cuda_ivf_stats;

/* ---- errors ---------------------------------------------------------------------------- */

/* Message of the last failed call on this thread, formatted like NNdexError's Display
 * (src/lib.rs:109-144). Never NULL; "" when the last call succeeded. */
NNDEX_API const char* nndex_cuda_last_error(void);

/* ---- devices --------------------------------------------------------------------------- */

/* Replaces gpu::list_gpu_devices (src/gpu.rs:992-1010). Writes up to `capacity` entries. */
NNDEX_API int nndex_cuda_list_devices(nndex_cuda_devinfo* out, uint32_t capacity, uint32_t* count);

/* Replaces NNdex::gpu_info (src/lib.rs:302-318). */
NNDEX_API int nndex_cuda_info(const nndex_cuda_index* index, nndex_cuda_devinfo* out);

/* ---- lifetime -------------------------------------------------------------------------- */

/*
 * Replaces NNdex::new (src/lib.rs:185-278) + GpuIndex::new (src/gpu.rs:138-309).
 * `host_matrix` is the caller's raw row-major f32 matrix of `n_values` values, read during the
 * call only. Validation order is the reference's: shape (src/lib.rs:191, 433-442), then finite
 * values, then zero-norm rows (src/lib.rs:239-244, 461-553). Normalisation, padding to a
 * multiple of 8 dims and the low-precision copies are made on the device.
 */
NNDEX_API int nndex_cuda_create(const float* host_matrix, uint64_t n_values, uint64_t rows, uint64_t dims,
                      uint32_t flags, const nndex_cuda_opts* opts, nndex_cuda_index** out);

/* Same as nndex_cuda_create, but the raw matrix already lives in device memory on the
 * selected device (no host copy). The call first waits for all work on the device, so the matrix
 * may still be in the making on any stream when it is called. */
NNDEX_API int nndex_cuda_create_from_device(const float* device_matrix, uint64_t n_values, uint64_t rows,
                                  uint64_t dims, uint32_t flags, const nndex_cuda_opts* opts,
                                  nndex_cuda_index** out);

/* ---- streaming construction and file loading ----------------------------------------------
 * The reference reads a .npy / .npz / .parquet matrix into one host Vec<f32> (load_matrix_from_disk,
 * src/python_io.rs:80-377) and then calls NNdex::new (src/python_bindings.rs:69-86). These entry
 * points let a loader hand the rows over in pieces instead: every piece is copied into pinned
 * staging and uploaded while the next one is read, and K1 (validation, normalisation, padding,
 * low-precision copies) runs on the device per piece. The finished index is identical to
 * nndex_cuda_create on the concatenated values, with the same errors in the same order. */
typedef struct nndex_cuda_builder nndex_cuda_builder;

/* Starts an index of rows × dims (both > 0, else NNDEX_ERR_SHAPE_MISMATCH). */
NNDEX_API int nndex_cuda_builder_begin(uint64_t rows, uint64_t dims, uint32_t flags, const nndex_cuda_opts* opts,
                             nndex_cuda_builder** out);
/* Appends the next `n_values` row-major values (any count, need not end on a row). Appending past
 * rows × dims fails with NNDEX_ERR_SHAPE_MISMATCH; the builder then only accepts finish/abort. */
NNDEX_API int nndex_cuda_builder_append(nndex_cuda_builder* builder, const float* host_values, uint64_t n_values);
/* Completes the index (shape check, then the first non-finite / zero-norm row, then the IVF when
 * approximate) and frees the builder, whatever the outcome. */
NNDEX_API int nndex_cuda_builder_finish(nndex_cuda_builder* builder, nndex_cuda_index** out);
/* Frees an unfinished builder. NULL is ignored. */
NNDEX_API void nndex_cuda_builder_abort(nndex_cuda_builder* builder);

/* Replaces load_npy + NNdex::new (src/python_io.rs:112-120): a little-endian float32, C-order,
 * 2-D .npy file (format 1.0-3.0), memory-mapped and streamed through the builder. Other .npy
 * layouts fail with NNDEX_ERR_INVALID_ARGUMENT ("failed to read .npy matrix from ..."); a 0-row or
 * 0-column array with NNDEX_ERR_SHAPE_MISMATCH ("matrix loaded from ... is empty or has zero
 * dimensions", src/python_io.rs:75-76). */
NNDEX_API int nndex_cuda_create_from_npy(const char* path, uint32_t flags, const nndex_cuda_opts* opts,
                               nndex_cuda_index** out);

/* Rust `Drop` for CudaIndex. NULL is ignored. */
NNDEX_API void nndex_cuda_destroy(nndex_cuda_index* index);

NNDEX_API int nndex_cuda_rows(const nndex_cuda_index* index, uint64_t* rows, uint64_t* dims,
                    uint64_t* padded_dims);

/* ---- search ---------------------------------------------------------------------------- */

/*
 * Replaces NNdex::search (src/lib.rs:335-355) → GpuIndex::search (src/gpu.rs:321-349).
 * Checks k > 0 (InvalidTopK) before query_len == dims (QueryDimensionalityMismatch), as the
 * reference does. Writes capped_k = min(k, rows) results (fewer only in approx mode when the
 * probed lists hold fewer rows; `count_out` receives the number written).
 */
NNDEX_API int nndex_cuda_search(nndex_cuda_index* index, const float* host_query, uint64_t query_len,
                      uint64_t k, uint64_t* idx_out, float* sim_out, uint64_t* count_out);

/*
 * Replaces NNdex::search_batch (src/lib.rs:372-402) → GpuIndex::search_batch
 * (src/gpu.rs:372-399). Checks the shape (ShapeMismatch) before k > 0 (InvalidTopK), as the
 * reference does. Outputs are row-major [query_rows × min(k, rows)]; `counts_out[q]` holds the
 * number of valid results of query q. Unused slots are (0, 0.0f), the padding
 * batch_neighbors_to_numpy applies (src/python_bindings.rs:477-483).
 */
NNDEX_API int nndex_cuda_search_batch(nndex_cuda_index* index, const float* host_queries,
                            uint64_t n_values, uint64_t query_rows, uint64_t k,
                            uint64_t* idx_out, float* sim_out, uint64_t* counts_out);

/*
 * Device-resident variant of nndex_cuda_search_batch: queries and outputs are device pointers
 * on the index's device, the work is enqueued on `stream` (a cudaStream_t, NULL = the legacy
 * default stream) after any earlier call's work on this index, and the call returns once it is
 * enqueued when `synchronize` is 0. Query
 * validation (finite, zero-norm) is reported through the returned status only when
 * `synchronize` is 1; otherwise through nndex_cuda_stream_status after the stream drains.
 */
NNDEX_API int nndex_cuda_search_batch_device(nndex_cuda_index* index, const float* dev_queries,
                                   uint64_t query_rows, uint64_t query_dims, uint64_t k,
                                   uint64_t* dev_idx_out, float* dev_sim_out,
                                   uint32_t* dev_counts_out, void* stream, int synchronize);

/*
 * Selects the scan precision for later searches (NNDEX_PRECISION_*; BF16/FP8 need the index to have
 * been created with NNDEX_FLAG_BF16/FP8) and the candidate width k' of the low-precision scan
 * (0 = autotuned). Low-precision searches return the exact FP32 top-k: the k' candidates are
 * re-scored in FP32 and queries whose exactness certificate fails are re-run on the FP32 scan.
 * Tensor-core searches synchronise the stream (the certificate's fallback is decided on the host).
 */
NNDEX_API int nndex_cuda_set_precision(nndex_cuda_index* index, uint32_t precision, uint32_t rerank_width);

/*
 * Candidates of the last exact low-precision search on this index (paths 2, 3 and 6; diagnostics
 * and error reports):
 * for each of `query_rows` queries, the k' rows ranked by approximate (BF16/FP8) score, with those
 * approximate scores, the bound eps the exactness certificate used for this index's copy (max row
 * residual) and, per query, whether its certificate held (0 = re-run on the FP32 scan). Host
 * buffers of query_rows × k' entries (certified_out: query_rows); *kprime receives k'.
 */
NNDEX_API int nndex_cuda_last_candidates(nndex_cuda_index* index, uint64_t query_rows, uint64_t* idx_out,
                                         float* approx_out, uint64_t capacity, uint32_t* kprime,
                                         float* eps_rows, uint32_t* certified_out);

/* Status word of the last asynchronous device call on this index (0 when clean). */
NNDEX_API int nndex_cuda_stream_status(nndex_cuda_index* index);

/* Statistics of the last search call on this index. */
NNDEX_API int nndex_cuda_last_search_stats(const nndex_cuda_index* index, nndex_cuda_search_stats* out);

/*
 * Kernel timing for roofline reports: while enabled, the library brackets every launch of the
 * dominant scan kernel with CUDA events on the stream it launches on. nndex_cuda_scan_timing
 * waits for the recorded events and returns their summed duration and count, then clears them.
 */
NNDEX_API int nndex_cuda_set_scan_timing(nndex_cuda_index* index, int enable);
NNDEX_API int nndex_cuda_scan_timing(nndex_cuda_index* index, double* total_ms, uint64_t* launches);

/* Total kernels this library has launched in this process (all indexes, all devices). */
NNDEX_API uint64_t nndex_cuda_kernel_launch_count(void);

/* ---- search without allocation -------------------------------------------------------- */

/* Size of the device array nndex_cuda_search_batch_device_noalloc works in (per GPU). */
#define NNDEX_NOALLOC_SCRATCH_BYTES (16u << 20)

/*
 * Exact batch search that allocates no memory; no counterpart in the reference. For callers that
 * cannot call cudaMalloc while searching: a process whose HBM is fully reserved by another
 * allocator, or a latency-critical path that cannot take cudaMalloc/cudaFree's implicit
 * synchronisation. Same arguments, results and validation as nndex_cuda_search_batch_device with
 * synchronize = 1 (it returns after the results are written). Its scratch memory is one
 * file-scope device array of NNDEX_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds
 * until exit; a batch whose normalised queries and candidate keys do not fit is rejected with
 * NNDEX_ERR_UNSUPPORTED (batches above 16,384 queries run in pieces of 16,384, each of which must
 * fit). Creating an index binds the array on the index's device (with lazy module loading that is
 * when the GPU takes its memory), so a search never does. All calls share the array: calls that
 * overlap on the GPU race. Indexes that answer through an IVF (NNDEX_FLAG_APPROX) are rejected
 * with NNDEX_ERR_UNSUPPORTED.
 */
NNDEX_API int nndex_cuda_search_batch_device_noalloc(nndex_cuda_index* index, const float* dev_queries,
                                                     uint64_t query_rows, uint64_t query_dims, uint64_t k,
                                                     uint64_t* dev_idx_out, float* dev_sim_out,
                                                     uint32_t* dev_counts_out, void* stream);

/* ---- IVF layout (approximate mode) --------------------------------------------------------- */

/*
 * The IVF built for an index created with NNDEX_FLAG_APPROX, as ApproxIndex holds it
 * (src/approx.rs:11-25). *nlist_out is always written (0 = no IVF: the index answers approx
 * searches exactly, as the reference does when the IVF gives no speedup, src/cpu.rs:399-407).
 * Each array may be NULL; otherwise it must hold: centroids nlist × padded_dims floats,
 * offsets nlist + 1, original_indices rows, init_rows nlist (the rows k-means++ picked).
 */
NNDEX_API int nndex_cuda_ivf_layout(nndex_cuda_index* index, uint64_t* nlist_out, float* centroids,
                                    uint64_t* offsets, uint64_t* original_indices, uint64_t* init_rows);
NNDEX_API int nndex_cuda_ivf_stats_get(const nndex_cuda_index* index, nndex_cuda_ivf_stats* out);
/*
 * Installs a saved IVF instead of building one (the build, src/approx.rs:46-100, is the most
 * expensive one-off of approximate mode). The arrays are the ones nndex_cuda_ivf_layout exports
 * from an index over the same matrix: centroids [nlist × padded_dims] f32, offsets [nlist + 1],
 * original_indices [rows] (reordered position → row), init_rows [nlist] or NULL. nlist 0 installs
 * "no IVF" (the reference answers such indexes exactly). Checks offsets (0 … rows, non-decreasing),
 * that original_indices is a permutation and that the centroids are finite
 * (NNDEX_ERR_INVALID_ARGUMENT otherwise); it cannot check that the layout was made from THIS
 * matrix: compare nndex_cuda_base_checksum values for that. Afterwards the index is in approximate
 * mode and answers as the index the layout was exported from. Waits for the device; not while a
 * server runs on the index.
 */
NNDEX_API int nndex_cuda_ivf_restore(nndex_cuda_index* index, uint64_t nlist, const float* centroids,
                                     const uint64_t* offsets, const uint64_t* original_indices,
                                     const uint64_t* init_rows);

/* 64-bit fingerprint of the stored (validated, normalised, padded) rows: Σ over positions i of
 * splitmix64(i · 2^32 + bits of value i), mod 2^64. Equal matrices give equal values on any GPU. */
NNDEX_API int nndex_cuda_base_checksum(nndex_cuda_index* index, uint64_t* checksum);

/* CUDA graphs for nndex_cuda_search / nndex_cuda_search_batch (on by default): the per-batch
 * sequence of an exact FP32 or IVF list-scan batch (status resets, query upload, prep, scan, merge,
 * result download) is captured the second time a (path, batch size, k) shape comes in a row and
 * replayed as one launch afterwards; results are identical either way. Any reallocation of a
 * scratch buffer, nndex_cuda_set_precision, nndex_cuda_set_nprobe or nndex_cuda_ivf_restore drops
 * the cached graphs. enable = 0 turns capture off (and drops them). */
NNDEX_API int nndex_cuda_set_graphs(nndex_cuda_index* index, int enable);

/*
 * The autotuner (replaces src/profiles.rs:65-185, which maps a shape to a CPU strategy by fixed
 * thresholds). mode 1 (the default): the first batch of each shape — exact or IVF, queries and k
 * rounded up to powers of two, nprobe and precision — runs every plan that returns the same
 * results (the FP32 scan or the TF32 candidate scan for small batches; BF16 or FP8 tensor-core
 * scans with pass-1 tile strides 1, 8 and 32 for large ones; the FP32 or the tensor-core IVF list
 * scan, the latter with pass-1 strides 1, 2, 4 and 16), times each, and keeps the fastest for later
 * batches of that shape. mode 0: the fixed
 * rules. mode 2: the cached plans, and the rules for shapes not in the cache (no batch pays for
 * measurements; the serving loop's slots run so, with the cache the index had when the server
 * started). Results are identical under every plan; only speed differs.
 */
NNDEX_API int nndex_cuda_set_autotune(nndex_cuda_index* index, int mode);
/*
 * The tuner's cache as text, to keep across processes: a header line naming the device, the
 * matrix shape and flags, then one line per shape with its plan and time. *len receives the size
 * (with the terminating 0); with buf NULL or too small only *len is written
 * (NNDEX_ERR_INVALID_ARGUMENT when buf is too small).
 */
NNDEX_API int nndex_cuda_autotune_export(nndex_cuda_index* index, char* buf, uint64_t capacity, uint64_t* len);
/* Installs a cache exported for the same device model, shape and flags (NNDEX_ERR_INVALID_ARGUMENT
 * otherwise: a plan measured elsewhere is not trusted). Replaces entries of the same shapes. */
NNDEX_API int nndex_cuda_autotune_import(nndex_cuda_index* index, const char* text);
/* Parses exported text without an index or a GPU: NNDEX_OK and the entry count, or
 * NNDEX_ERR_INVALID_ARGUMENT and the first bad line in the error message. */
NNDEX_API int nndex_cuda_autotune_validate(const char* text, uint64_t* entries);

/* Lists probed per query by later approx searches (0 = choose_nprobe, src/approx.rs:318-336);
 * no counterpart in the reference, whose nprobe is always the policy's. */
NNDEX_API int nndex_cuda_set_nprobe(nndex_cuda_index* index, uint32_t nprobe);

/* ---- serving: continuous batching (replaces the query caches, src/cpu.rs:16-89, src/gpu.rs:21-25) ----
 *
 * A server owns `slots` views of one index (each: its own stream and scratch, the index's device
 * data shared) and one worker thread per slot. Submitted requests wait in a queue; whenever a slot
 * is free its worker takes every queued request of the same kind (exact, or approx with the same
 * nprobe) that fits the slot, in arrival order, and runs them as one batch at their largest k (each
 * request receives its own k; a query's result does not depend on the batch it ran in). Requests
 * that arrive while batches are on the GPU join the next batch of the first slot to free up; slots
 * run concurrently on the device.
 * Admission by memory: every slot may hold at most `slot_bytes` of per-batch device memory
 * (0 = free HBM × 0.5 / slots at start), estimated per query from k; a request that cannot fit a
 * slot, or that would take the queue above `queue_capacity` queries, is refused with
 * NNDEX_ERR_ADMISSION (the caller may retry later). The index must outlive its servers.
 */
typedef struct nndex_cuda_server nndex_cuda_server;
typedef struct nndex_cuda_server_opts {
    uint32_t slots;              /* concurrent batches (worker threads), 0 = 2                  */
    uint32_t max_batch_queries;  /* queries per batch, 0 = 4096                                 */
    uint64_t queue_capacity;     /* queries waiting, 0 = 1 << 20                                */
    uint64_t slot_bytes;         /* device memory per slot, 0 = free HBM × 0.5 / slots          */
    uint32_t latency_budget_ms;  /* refuse a request while the oldest queued request has waited
                                    longer than this (the queue is backed up), 0 = no latency
                                    bound                                                        */
    uint32_t reserved[7];
} nndex_cuda_server_opts;
typedef struct nndex_cuda_request_info {
    uint64_t submit_ns, start_ns, done_ns;   /* steady-clock times: queued, batch launched, done */
    uint64_t batch_id;
    uint32_t batch_queries;                  /* queries in the batch it ran in                  */
    uint32_t slot;
    uint32_t path;                           /* nndex_cuda_search_stats::path of the batch      */
    uint32_t reserved;
} nndex_cuda_request_info;
typedef struct nndex_cuda_server_stats {
    uint64_t requests_done, queries_done, batches, refused;
    uint64_t queued_queries, max_queued_queries;
    uint32_t slots, max_batch_queries;
    uint64_t slot_bytes;
    uint64_t refused_latency;      /* of `refused`: refused by the latency budget               */
    double us_per_query;           /* moving average of a slot's wall time per query (batches'
                                      launch to results), for reports                           */
    uint64_t fp32_fallback_queries;  /* queries of all batches re-run on an FP32 scan            */
    double slowest_batch_ms;         /* the slowest batch so far: its wall time,                */
    uint32_t slowest_batch_queries;  /*   its queries,                                           */
    uint32_t slowest_batch_k;        /*   the k it ran at,                                       */
    uint32_t slowest_batch_path;     /*   its path (nndex_cuda_search_stats::path)               */
    uint32_t slowest_batch_approx;   /*   and whether it was an IVF batch                        */
} nndex_cuda_server_stats;

NNDEX_API int nndex_cuda_server_start(nndex_cuda_index* index, const nndex_cuda_server_opts* opts,
                                      nndex_cuda_server** out);
/* Queues `query_rows` raw queries (copied before the call returns). flags: NNDEX_FLAG_APPROX for
 * an IVF search (the index must have one; otherwise the request is answered exactly, as the
 * reference does). nprobe: 0 = the index's setting. */
NNDEX_API int nndex_cuda_server_submit(nndex_cuda_server* server, const float* host_queries,
                                       uint64_t query_rows, uint64_t query_dims, uint64_t k,
                                       uint32_t flags, uint32_t nprobe, uint64_t* ticket);
/* NNDEX_OK with the results (idx/sim: query_rows × min(k, rows); counts: query_rows) once the
 * request has finished (the ticket is then retired), NNDEX_PENDING if it has not within
 * `timeout_ms` (0 = do not wait, negative = wait until it finishes), or the request's error. */
NNDEX_API int nndex_cuda_server_poll(nndex_cuda_server* server, uint64_t ticket, int32_t timeout_ms,
                                     uint64_t* idx_out, float* sim_out, uint64_t* counts_out,
                                     nndex_cuda_request_info* info);
NNDEX_API int nndex_cuda_server_stats_get(nndex_cuda_server* server, nndex_cuda_server_stats* out);
/* Finishes the queued requests, joins the workers and frees the slots. */
NNDEX_API void nndex_cuda_server_stop(nndex_cuda_server* server);

/* ---- failure handling checks (no counterpart in the reference, whose GPU waits have no limit:
 * src/gpu.rs:573, 756) ------------------------------------------------------------------------ */

/* Runs one bounded device wait, of `budget_cycles` clock cycles (1 .. 2e9), on an mbarrier that
 * nothing completes: the kernel records a timeout status and returns, and the call reports it as
 * NNDEX_ERR_TIMEOUT like any search whose wait ran out. The index stays usable afterwards. */
NNDEX_API int nndex_cuda_check_bounded_wait(nndex_cuda_index* index, uint64_t budget_cycles);

/* Fault injection on the host: the next `count` scratch or staging allocations made by any index
 * fail as if the GPU were out of memory (no cudaMalloc is attempted), and the calls that needed them
 * return NNDEX_ERR_OUT_OF_MEMORY. 0 cancels. For tests of callers' out-of-memory handling. */
NNDEX_API void nndex_cuda_inject_alloc_failures(uint32_t count);

/* ---- launch planning (host only: no GPU, no index) ------------------------------------------ */

/* The row ranges the tensor-core scan splits `rows` rows into for `groups` CTAs per range (its
 * 128-query blocks, or the two CTAs of a pair per pair) on `sm_count` SMs, one CTA per SM at a
 * time: *range_rows (a multiple of 256, at least 2,048 rows unless the base is smaller) and
 * *nranges minimise ceil(groups × nranges / sm_count) × the tiles of a range over 1 to 8 rounds. */
NNDEX_API int nndex_cuda_plan_tc_ranges(uint64_t rows, uint64_t groups, uint32_t sm_count, uint64_t* nranges,
                                        uint64_t* range_rows);
/* The FP32 scan's grid for `nq` queries at `k` over `rows` stored rows of `dims` values on
 * `sm_count` SMs with `smem_limit` bytes of shared memory per block: *qb queries per CTA, *groups
 * query groups and *ctas_per_group CTAs per group (each a contiguous share of the rows). */
NNDEX_API int nndex_cuda_plan_fp32_scan(uint32_t nq, uint32_t dims, uint32_t k, uint64_t rows, uint32_t sm_count,
                                        uint64_t smem_limit, uint32_t* qb, uint32_t* groups,
                                        uint32_t* ctas_per_group);

/* ---- FP64 oracle on the device (score-error report) ------------------------------------- */

/*
 * For `n` (query, row) pairs, computes the FP64 dot product of the stored (normalised, FP32)
 * row with the query as normalised by the index (so the result is the exact score the FP32 path
 * approximates). `dev_*` are device pointers; `rows_idx` are row indices into the index.
 */
NNDEX_API int nndex_cuda_fp64_scores(nndex_cuda_index* index, const float* dev_queries_normalized,
                           uint64_t query_rows, const uint64_t* dev_pairs_query,
                           const uint64_t* dev_pairs_row, uint64_t n, double* dev_out);

/*
 * Per-result score errors (no counterpart in the reference, whose results carry no error): while
 * enabled, every search also scores each returned (query, row) pair in FP64 on the device — the
 * stored FP32 row against the query as the index normalised it, the exact value the returned FP32
 * score approximates — and records |returned score − FP64 score| per result. The extra work is one
 * FP64 dot product per result. The no-allocation entry point records none. Enabling or disabling
 * drops the cached CUDA graphs (and the host-buffer search is not captured while enabled).
 */
NNDEX_API int nndex_cuda_set_error_report(nndex_cuda_index* index, int enable);
/*
 * The last search's per-result errors: query_rows × min(k, rows) doubles in result order (0 where a
 * query returned fewer results). query_rows and k must be the last search's. Waits for the search.
 */
NNDEX_API int nndex_cuda_last_score_errors(nndex_cuda_index* index, uint64_t query_rows, uint64_t k,
                                           double* errors_out);

#ifdef __cplusplus
}
#endif

#endif /* NNDEX_CUDA_H */
