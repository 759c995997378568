// index.h — the CUDA backend object behind the C ABI (one per NNdex built with the Cuda backend).
#pragma once

#include <memory>
#include <map>
#include <mutex>
#include <unordered_map>
#include <utility>
#include <vector>

#include "internal.h"
#include "ivf.h"

namespace nndex {

// Queries handled per scan launch sequence; larger batches are processed in chunks.
constexpr uint64_t kMaxBatchChunk = 16384;
// Rows a pass-2 query may collect before it is re-run on the FP32 scan.
constexpr uint32_t kSecondPassCap = 8192;

// Incremented whenever a scratch or staging buffer of any index is (re)allocated: a captured
// CUDA graph is valid only while the epoch it was captured in lasts.
uint64_t alloc_epoch();
void bump_alloc_epoch();
// Host-side fault injection (tests): the next n scratch allocations fail as out of memory.
void inject_alloc_failures(uint32_t n);
bool take_injected_alloc_failure();
// Scratch growth. By default a buffer that must grow is freed with cudaFree (which waits for the
// whole device) and reallocated with cudaMalloc. A serving slot instead grows its buffers in
// stream order on its own stream (cudaFreeAsync / cudaMallocAsync), so a slot meeting a larger
// batch does not wait for the batches the other slots are running; every buffer it grows is then
// stream-ordered memory from the start (a slot is a fresh view). The stream is per thread.
void set_scratch_stream(cudaStream_t s);
cudaStream_t scratch_stream();
// Frees `p` and allocates `bytes` (0 → 1) into it under the current thread's growth mode.
cudaError_t regrow_raw(void** p, size_t bytes);

int set_error(int code, const char* fmt, ...);
int last_encode_result();  // CUresult of this thread's last tensor-map encode
void clear_error();
const char* last_error();
int cuda_error(cudaError_t e, const char* what);
// NNdexError::ShapeMismatch (src/lib.rs:109-112).
int err_shape(uint64_t rows, uint64_t dims, uint64_t values);

struct CudaIndex {
    bool owns_base = true;    // false for a view (make_view): the device data belongs to another handle
    int device = 0;
    int sm_count = 148;
    size_t smem_optin = 232448;
    uint64_t rows = 0;        // stored rows
    uint64_t rows_alloc = 0;  // rows rounded up to 128 (zero rows beyond `rows`)
    uint64_t dims = 0;        // caller dimensionality
    uint64_t dp = 0;          // nndex padded_dims (multiple of 8, src/lib.rs:192)
    uint64_t ds = 0;          // device row stride: dims rounded up to 32 floats (one 128 B TMA slab)
    uint32_t flags = 0;
    bool normalized = false;
    bool approx = false;
    nndex_cuda_opts opts{};

    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t done_ev = nullptr;        // completion of the last call's device work
    cudaStream_t done_stream = nullptr;   // the stream it ran on
    std::mutex mu;

    float* d_base = nullptr;  // rows_alloc × ds FP32, normalised, zero padded
    CUtensorMap tmap_f32{};
    CUtensorMap tmap_f32_176{};  // box {32 floats, 176 rows}: the 11-warp wide FP32 scan's tiles
    CUtensorMap tmap_f32_112{};  // box {32 floats, 112 rows}: the 7-warp wide FP32 scan's tiles

    // Low-precision scoring copies (NNDEX_FLAG_BF16 / NNDEX_FLAG_FP8), K3.
    uint32_t precision = NNDEX_PRECISION_AUTO;
    uint64_t kb16 = 0;                         // BF16 row length: dims rounded up to 64
    uint64_t kf8 = 0;                          // FP8 row length: dims rounded up to 128
    __nv_bfloat16* d_base_bf16 = nullptr;      // rows_alloc × kb16
    uint8_t* d_base_fp8 = nullptr;             // rows_alloc × kf8 (E4M3)
    float* d_row_scale = nullptr;              // rows_alloc: FP8 dequantisation scale per row
    float2* d_tile_scale = nullptr;            // rows_alloc / 256: FP8 {min, max} scale per 256-row tile
    float eps_bf16 = 0.0f, eps_fp8 = 0.0f;     // max row residual norm ‖x − x̂‖
    float* d_res16 = nullptr;                  // rows: ‖x − x̂‖ of the BF16 copy
    float* d_res8 = nullptr;                   // rows: ‖x − x̂‖ of the FP8 copy
    CUtensorMap tmap_bf16{}, tmap_fp8{};
    CUtensorMap tmap_bf16_h{}, tmap_fp8_h{};   // the same with 128-row boxes (two-block pass 2)
    // per-search buffers of the tensor-core path
    __nv_bfloat16* d_q_bf16 = nullptr;
    size_t cap_q_bf16 = 0;
    uint8_t* d_q_fp8 = nullptr;
    size_t cap_q_fp8 = 0;
    float* d_q_scale = nullptr;
    size_t cap_q_scale = 0;
    float2* d_tfnorm = nullptr;  // K12: per row {‖x‖, ‖x − tf32_head(x)‖}, rounded up (shared by views)
    float* d_q_resid = nullptr;
    size_t cap_q_resid = 0;
    unsigned long long* d_thr = nullptr;
    size_t cap_thr = 0;
    uint64_t* d_cand_idx = nullptr;
    size_t cap_cand_idx = 0;
    float* d_cand_sim = nullptr;
    size_t cap_cand_sim = 0;
    uint32_t* d_cand_cnt = nullptr;
    size_t cap_cand_cnt = 0;
    uint32_t* d_cert = nullptr;
    size_t cap_cert = 0;
    uint32_t* h_cert = nullptr;
    size_t cap_hcert = 0;
    float* d_qsub = nullptr;  // FP32 queries re-run after a failed certificate
    size_t cap_qsub = 0;
    uint64_t* d_fb_idx = nullptr;  // their FP32 results before they move to the query's slots
    size_t cap_fb_idx = 0;
    float* d_fb_sim = nullptr;
    size_t cap_fb_sim = 0;
    uint32_t* d_fb_cnt = nullptr;
    size_t cap_fb_cnt = 0;
    uint32_t last_tc_n = 0;  // queries of the last tensor-core batch (diagnostics)
    uint32_t tc_sample_stride = 1;  // pass-1 tile stride by the certification rule (1 = full pass 1)
    uint32_t forced_stride = 0;     // the tuned plan's pass-1 tile stride for the current batch (0 = rule)
    uint32_t forced_qb = 0;         // the tuned plan's pass-2 query blocks per CTA (0 = rule)
    uint32_t last_tc_stride = 1;
    float* d_kth = nullptr;  // pass 1: exact k-th score per query
    unsigned long long* d_floor = nullptr;  // TF32 scan: per query, a key its k'-th candidate reaches
    size_t cap_floor = 0;
    uint64_t* d_rslots = nullptr;  // pass 2: each rerank work item's best k keys
    size_t cap_rslots = 0;
    size_t cap_kth = 0;
    // pass 2 (threshold collection) buffers
    uint32_t* d_ids = nullptr;
    size_t cap_ids = 0;
    uint8_t* d_q2_lp = nullptr;
    size_t cap_q2_lp = 0;
    float* d_q2_resid = nullptr;
    size_t cap_q2_resid = 0;
    float* d_q2_scale = nullptr;
    size_t cap_q2_scale = 0;
    float* d_q2_thr = nullptr;
    size_t cap_q2_thr = 0;
    uint32_t* d_rows2 = nullptr;
    size_t cap_rows2 = 0;
    uint32_t* d_cnt2 = nullptr;
    size_t cap_cnt2 = 0;
    uint32_t* d_ok2 = nullptr;
    size_t cap_ok2 = 0;
    uint32_t* h_ids = nullptr;
    size_t cap_hids = 0;
    uint32_t* h_ok2 = nullptr;
    size_t cap_hok2 = 0;
    uint32_t rerank_width = 0;  // k′ override (0 = autotuned)


    // per-search buffers (grown on demand)
    float* d_qraw = nullptr;
    size_t cap_qraw = 0;
    float* d_qn = nullptr;
    size_t cap_qn = 0;
    uint64_t* d_ws = nullptr;
    size_t cap_ws = 0;
    // Results of the host-buffer search: idx (n·k u64), sim (n·k f32) and cnt (n u32) laid out
    // back to back in one device buffer and one pinned buffer, so a single copy downloads them
    // (ensure_result_capacity sets the three views for the batch's shape).
    uint8_t* d_res = nullptr;
    size_t cap_res = 0;
    uint8_t* h_res = nullptr;
    size_t cap_hres = 0;
    uint64_t* d_idx = nullptr;
    float* d_sim = nullptr;
    uint32_t* d_cnt = nullptr;
    uint64_t* h_idx = nullptr;
    float* h_sim = nullptr;
    uint32_t* h_cnt = nullptr;
    size_t res_bytes = 0;        // bytes of the current batch's results
    // Status words, adjacent in one 16-byte allocation (d_status = the word after d_err), read back
    // with one copy into h_flags.
    unsigned long long* d_err = nullptr;
    uint32_t* d_status = nullptr;
    float* h_q = nullptr;
    size_t cap_hq = 0;
    uint64_t* h_flags = nullptr;

    // split cross-CTA merge (merge_topk_kernel with several blocks per query)
    uint64_t* d_part_keys = nullptr;
    size_t cap_part_keys = 0;
    uint32_t* d_part_done = nullptr;
    size_t cap_part_done = 0;
    int merge_workspace(uint64_t per_query, uint32_t nq, uint32_t k, MergeArgs& m, cudaStream_t s);

    nndex_cuda_search_stats stats{};
    std::shared_ptr<const IvfIndex> ivf;  // approximate mode (NNDEX_FLAG_APPROX), built at creation
    IvfScratch ivf_scratch;
    int approx_override = -1;   // -1: the index's mode; 0: exact; 1: approx (server batches)

    // CUDA graphs of the host-buffer search: the whole per-batch sequence (status resets, query
    // upload, query prep, scan, merge, result downloads) works on buffers this index owns, so a
    // shape seen twice in a row is captured once and replayed as one launch. A graph is dropped
    // when any scratch buffer has been reallocated since its capture (alloc_epoch()).
    struct GraphEntry {
        int path = 0, mode = 0;
        uint64_t n = 0, kcap = 0, epoch = 0;
        uint32_t nprobe = 0;  // the IVF scan's probe count at capture (0: chosen per batch)
        cudaGraphExec_t exec = nullptr;
        nndex_cuda_search_stats stats{};
        uint64_t launches = 0;
    };
    std::vector<GraphEntry> graphs;
    GraphEntry graph_seen;          // the last shape run without a graph (capture candidate)
    bool use_graphs = true;
    uint32_t graph_failed_paths = 0;  // paths whose capture failed (not tried again)
    void drop_graphs();

    // per-result score errors (nndex_cuda_set_error_report): |result − FP64 score| per result of the
    // last call, and {max as double bits, sum, count} for its statistics
    bool error_report = false;
    double* d_serr = nullptr;
    size_t cap_serr = 0;
    unsigned long long* d_serr_acc = nullptr;
    unsigned long long* h_serr_acc = nullptr;  // pinned copy of d_serr_acc
    uint64_t serr_nq = 0, serr_k = 0, serr_off = 0;  // the last call's shape; the current piece's first query
    cudaStream_t serr_stream = nullptr;
    bool serr_pending = false;  // statistics not yet read back
    int serr_begin(uint64_t nq, uint64_t kcap, cudaStream_t s);
    void serr_record(uint32_t n, uint32_t kcap, const uint64_t* idx, const float* sim, const uint32_t* cnt,
                     cudaStream_t s);
    int serr_fetch_stats();

    // Counters a device-side certificate fallback leaves on the device ({queries re-run on the FP32
    // scan, spare}), read back with the statistics.
    uint32_t* d_fbq = nullptr;  // the re-run queries' indices
    size_t cap_fbq = 0;
    uint32_t* d_fbn = nullptr;  // {TF32 re-runs, TC pass-2 queries, TC pass-2 overflows, spare}
    uint32_t* h_fbn = nullptr;  // pinned copy
    uint32_t* d_tcfail = nullptr;  // TC pass 2: positions (in d_ids) of the queries whose collection overflowed
    size_t cap_tcfail = 0;
    int ensure_fbn();
    cudaStream_t fbn_stream = nullptr;
    bool fbn_pending = false;
    int fetch_fallback_stats();

    // scan-kernel timing (roofline reports)
    bool scan_timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> scan_events;
    size_t scan_events_used = 0;
    void scan_event_begin(cudaStream_t s, cudaEvent_t& a);
    void scan_event_end(cudaStream_t s, cudaEvent_t a);

    ~CudaIndex();
    int ensure_query_capacity(uint64_t nq);
    int ensure_result_capacity(uint64_t nq, uint64_t kcap);
    int enqueue_query_prep(uint64_t nq, int mode, cudaStream_t s);
    int enqueue_exact_fp32(const float* d_queries, uint32_t nq, uint32_t k, uint32_t out_stride, uint64_t* o_idx,
                           float* o_sim, uint32_t* o_cnt, cudaStream_t s);
    int check_device_words();
    int search_host(const float* queries, uint64_t nq, uint64_t k, int mode, uint64_t* idx_out, float* sim_out,
                    uint64_t* counts_out);
    int search_device(const float* d_queries, uint64_t nq, uint64_t k, uint64_t* d_idx_out, float* d_sim_out,
                      uint32_t* d_cnt_out, cudaStream_t s, int synchronize);
    int run_device_chunk(const float* dq, uint64_t n, uint64_t kcap, int path, uint64_t* oi, float* os,
                         uint32_t* oc, cudaStream_t s, bool* synced);
    // Path choice for a batch: 1 = FP32 scan, 2 = BF16 tensor-core scan, 3 = FP8 tensor-core scan,
    // 6 = TF32 tensor-core candidate scan + exact FP32 rerank (small batches of an FP32 index).
    int choose_path(uint64_t nq, uint64_t kcap) const;
    // K12's plan for k results: candidates per query and CTA (0: no plan), buffer, ring depth.
    struct Tf32Plan {
        uint32_t kp = 0;      // candidates per query after the merge (k′)
        uint32_t kp_cta = 0;  // candidates per query and CTA
        uint32_t cap = 0, stages = 0;
    };
    Tf32Plan plan_tf32(uint64_t nq, uint64_t kcap) const;
    float tf32_c_norm() const;  // C of K12's bound: ε = ‖q‖(‖d_x‖ + C‖x‖) + ‖d_q‖(‖x‖ + ‖d_x‖)
    float tf32_eps() const;     // the largest ε for unit rows and queries
    int ivf_path(uint64_t nq, uint64_t kcap) const;

    // Autotuner (autotune.cu): for each batch shape (exact or IVF, queries and k rounded up to
    // powers of two, nprobe, precision) the plans that return the same results are timed once on
    // the first batch of that shape, and the fastest is kept. A plan is a path and, for the
    // tensor-core scan, its pass-1 tile stride.
    struct TunePlan {
        int path = 0;
        uint32_t stride = 0;  // 0 = the certification rule
        uint32_t qb = 0;      // tensor-core pass 2: query blocks per CTA (1 or 2; 0 = the rule)
    };
    struct TuneEntry {
        TunePlan plan;
        double ms = 0.0;      // its wall time per batch when measured
        uint32_t candidates = 0;
    };
    int autotune = 1;  // 0 = rules only, 1 = measure once per shape, 2 = cached plans, else rules
    std::map<uint64_t, TuneEntry> tune_cache;
    uint64_t tune_key(uint64_t nq, uint64_t kcap) const;
    std::vector<TunePlan> tune_candidates(uint64_t nq, uint64_t kcap) const;
    TunePlan rule_plan(uint64_t nq, uint64_t kcap) const;
    // The plan for a batch: cached, or by the rules; *measure when the tuner should time the
    // candidates on this batch first.
    TunePlan plan_for(uint64_t nq, uint64_t kcap, bool* measure) const;
    // The first host-buffer batch of a shape: every candidate plan timed on it (the queries in h_q).
    int tune_host(uint64_t n, uint64_t kcap, int mode, TunePlan* plan);
    struct TcPlan {
        uint32_t kp = 0;        // pass-1 heap entries per query (0: no plan)
        uint32_t stages = 0;    // ring depth
        bool stream_a = false;  // query slabs staged per ring stage instead of resident
    };
    TcPlan plan_tc(uint64_t kcap, bool fp8) const;
    uint32_t tc_chunks(bool fp8) const;
    void tc_ranges(uint32_t nqb, uint64_t& nranges, uint64_t& range_rows) const;
    void fill_tc_params(bool fp8, uint32_t n, uint64_t range_rows, TcParams& p) const;
    int encode_query_tmap(bool fp8, void* buf, uint32_t n, CUtensorMap* map) const;
    int enqueue_prep_queries(const float* d_raw, uint64_t n, int mode, int path, cudaStream_t s);
    int enqueue_tc(bool fp8, uint32_t n, uint32_t kcap, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt,
                   cudaStream_t s);
    // Pass 2 of a tensor-core batch on the device, after enqueue_tc: the uncertified queries are
    // compacted and gathered, their rows collected against T and reranked, and the queries whose
    // collection overflowed compacted for the host (d_fbn[1..2], d_tcfail). No host round trip.
    int enqueue_tc_pass2(bool fp8, uint32_t n, uint32_t kcap, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt,
                         cudaStream_t s);
    // Once the stream has completed a tensor-core batch (h_fbn read back with it): statistics, the
    // pass-1 stride rule, and the FP32 re-run of any query whose collection overflowed (device
    // outputs patched in place; synchronises the stream again only then).
    int finish_tc(uint32_t n, uint32_t kcap, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt, cudaStream_t s);
    int enqueue_tf32(uint32_t n, uint32_t kcap, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt, cudaStream_t s);
    // The FP32 scan for the listed queries (rows of d_qn), written into their output slots.
    int rerun_exact_fp32(const std::vector<uint32_t>& qs, uint32_t kcap, uint64_t* o_idx, float* o_sim,
                         uint32_t* o_cnt, cudaStream_t s);
    int stream_status();
    int enqueue_host_batch(uint64_t n, uint64_t kcap, int mode, int path);
    int run_host_batch(uint64_t n, uint64_t kcap, int mode, int path);
    // Approximate mode with an IVF that gives a speedup (src/approx.rs:35-37 provides_speedup).
    bool uses_ivf() const {
        const bool want = approx_override < 0 ? approx : approx_override == 1;
        return want && ivf && rows >= 256 && ivf->nlist >= 4;
    }
    void order_after_previous(cudaStream_t s);
    void mark_done(cudaStream_t s);
};

int make_view(const CudaIndex& src, CudaIndex** out);
int index_begin(uint64_t rows, uint64_t dims, uint32_t flags, const nndex_cuda_opts* opts, CudaIndex** out);
void index_prep_rows(CudaIndex* ix, const float* d_src, uint64_t row0, uint64_t n);
int index_finish(CudaIndex* ix);  // deletes ix on failure
int search_device_noalloc(CudaIndex* ix, const float* d_queries, uint64_t nq, uint64_t k, uint64_t* d_idx_out,
                          float* d_sim_out, uint32_t* d_cnt_out, cudaStream_t s);
// Looks up the no-allocation array's address on `device` (current), which loads the module that
// holds it; index creation calls it so that the array's memory is taken then, not at a first search.
int noalloc_bind(int device);

}  // namespace nndex

// The opaque handle behind the C ABI.
struct nndex_cuda_index {
    nndex::CudaIndex* impl;
};
