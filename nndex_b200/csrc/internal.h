// internal.h — host-side declarations shared by the library's translation units.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/nndex_cuda.h"

namespace nndex {

// Number of kernels launched by this library (process-wide). Called after each launch; with
// NNDEX_SYNC_CHECK=1 in the environment it also waits for the device and prints the launch site of
// the first CUDA error to stderr (a debugging aid: every launch then runs alone).
void count_launch_at(const char* file, int line, uint32_t n);
constexpr uint32_t launches_of() { return 1; }
constexpr uint32_t launches_of(uint32_t n) { return n; }
#define count_launch(...) ::nndex::count_launch_at(__FILE__, __LINE__, ::nndex::launches_of(__VA_ARGS__))
bool sync_check_enabled();
// With the sync check on: a description of the next launch, printed with its error (cleared by
// count_launch).
void set_launch_note(const char* fmt, ...);
uint64_t kernel_launches_total();

struct PrepArgs {
    const float* src = nullptr;  // rows × dims raw values (device)
    uint64_t rows = 0;
    uint32_t dims = 0;
    uint64_t row_base = 0;       // global index of src row 0 (for error reporting)
    float* out = nullptr;        // rows × out_stride
    uint32_t out_stride = 0;
    int mode = 0;                // 0 normalize_rows, 1 normalize_vector, 2 finite check + pad
    unsigned long long* err = nullptr;  // (row << 8) | code, reduced with atomicMin
    __nv_bfloat16* out_bf16 = nullptr;
    uint32_t bf16_stride = 0;
    uint8_t* out_fp8 = nullptr;
    uint32_t fp8_stride = 0;
    float* fp8_scale = nullptr;
    float* resid_bf16 = nullptr;
    float* resid_fp8 = nullptr;
    int sm_count = 148;
};
void launch_prep_rows(const PrepArgs& a, cudaStream_t stream);

// FP32 exact scan (K2) + cross-CTA merge.
struct ScanPlan {
    uint32_t qb = 16;          // queries per CTA (1, 2, 4, 8, 16)
    uint32_t ctas_per_group = 148;
    uint32_t groups = 1;
    uint32_t cap = 512;        // candidate buffer capacity per query
    uint32_t stages = 4;
    size_t smem_bytes = 0;
    uint32_t wide = 0;         // 0, or the consumer warps of the wide scan (8 or 16)
};

struct ScanArgs {
    const CUtensorMap* tmap = nullptr;  // base fp32 rows × dp, box {32, 128}, 128B swizzle
    const CUtensorMap* tmap_tile = nullptr;  // the same rows, box {32, 176}: the 11-warp wide scan's tiles
    const CUtensorMap* tmap_112 = nullptr;   // the same rows, box {32, 112}: the 7-warp wide scan's tiles
    const float* queries = nullptr;     // nq × dq normalised, zero padded
    uint32_t nq = 0;
    uint32_t dq = 0;                    // multiple of 32
    uint64_t rows = 0;
    uint32_t k = 0;                     // capped k
    const uint32_t* row_map = nullptr;  // optional: stored position → original row index
    uint64_t* ws_keys = nullptr;        // nq × ctas_per_group × k
    uint32_t* status = nullptr;
    const uint32_t* live = nullptr;     // optional: a device count; 0 makes the whole launch return
};

// Picks queries-per-CTA, grid and candidate capacity for (nq, dq, k) within the shared-memory
// budget. Returns false when k is above what the fused kernel supports.
bool plan_scan_fp32(uint32_t nq, uint32_t dq, uint32_t k, uint64_t rows, int sm_count, size_t smem_limit,
                    ScanPlan& plan);
cudaError_t launch_scan_fp32(const ScanArgs& a, const ScanPlan& plan, cudaStream_t stream);

struct MergeArgs {
    const uint64_t* ws_keys = nullptr;  // nq × per_query candidate keys (0 = empty slot)
    uint32_t nq = 0;
    uint64_t per_query = 0;
    uint32_t k = 0;
    uint32_t out_stride = 0;            // result slots per query in the outputs
    uint64_t* idx_out = nullptr;        // nq × out_stride
    float* sim_out = nullptr;
    uint32_t* count_out = nullptr;      // nq
    // Optional split of each query's lists over several blocks (merge_parts(per_query, k, nq) of them):
    // part_keys holds nq × parts × k keys, part_done nq counters that start (and end) at zero.
    uint64_t* part_keys = nullptr;
    uint32_t* part_done = nullptr;
    const uint32_t* live = nullptr;     // optional: a device count; queries at or past it are skipped
    const uint32_t* out_rows = nullptr;  // optional: query q's results go to output row out_rows[q]
};
uint32_t merge_parts(uint64_t per_query, uint32_t k, uint32_t nq);
cudaError_t launch_merge_topk(const MergeArgs& a, cudaStream_t stream);

// K3 tensor-core scan (BF16 / FP8), two passes, and K4 rerank.

// Row ranges of a tensor-core scan grid of `groups` CTAs per range (its query blocks, or a pair's
// two CTAs per pair). One CTA fits an SM, and every range but the last holds the same number of
// 256-row tiles, so the launch takes ceil(groups × ranges / sms) rounds of one range's tiles: the
// split minimises that product over 1 to 8 rounds. (Four ranges per SM with 32 query blocks made
// 608 CTAs on 148 SMs: 4.1 rounds, the fifth with 16 CTAs and 132 SMs idle.) A range holds at
// least 2,048 rows. The host derives pass 1's grid with it, pass 2's CTAs from the live query count.
__host__ __device__ inline void tc_range_split(uint64_t rows, uint64_t groups, uint64_t sms, uint64_t& nranges,
                                               uint64_t& range_rows) {
    const uint64_t tiles = (rows + 255) / 256;
    if (tiles == 0 || groups == 0 || sms == 0) {
        nranges = 1;
        range_rows = 256;
        return;
    }
    uint64_t nr_max = (rows + 2047) / 2048;
    if (nr_max < 1) nr_max = 1;
    uint64_t best_tpr = tiles, best_cost = ~0ull;
    for (uint64_t m = 1; m <= 8; ++m) {
        uint64_t nr = m * sms / groups;
        nr = nr < 1 ? 1 : (nr > nr_max ? nr_max : nr);
        const uint64_t tpr = (tiles + nr - 1) / nr;  // tiles per range
        const uint64_t used = (tiles + tpr - 1) / tpr;
        const uint64_t cost = (groups * used + sms - 1) / sms * tpr;
        if (cost < best_cost) {  // ties keep the fewer rounds
            best_cost = cost;
            best_tpr = tpr;
        }
    }
    range_rows = best_tpr * 256;
    nranges = (rows + range_rows - 1) / range_rows;
}

struct TcParams {
    uint32_t nq = 0;
    uint32_t nchunks = 0;                 // K bytes / 128
    uint32_t kprime = 0;                  // pass 1: keys per (query, range or item) slot
    // pass 1 heap size (≤ kprime; the slot's rest is zero): kprime when pass 1 may certify; a
    // sampled pass 1 only has to yield T, for which each slot's best k suffice
    uint32_t heap_k = 0;
    uint32_t cap2 = 0;                    // pass 2 rows collected per query
    uint64_t rows = 0;
    uint64_t range_rows = 0;              // rows per CTA range (multiple of 256)
    uint32_t tile_stride = 1;             // scan every tile_stride-th 256-row tile (pass-1 sampling)
    const float* row_scale = nullptr;     // FP8 only
    const float2* tile_scale = nullptr;   // FP8 only: per 256-row tile, {min, max} of its rows' scales
    const float* q_scale = nullptr;       // FP8 only
    const float* row_resid = nullptr;     // ‖x − x̂‖ per row
    const float* q_resid = nullptr;       // ‖q − q̂‖ per query
    float eps_acc = 0.0f;                 // FP32 accumulation error bound
    float eps_rows = 0.0f;                // max ‖x − x̂‖ over the rows
    unsigned long long* thr_global = nullptr;  // pass 1: per query, zeroed before the launch
    uint64_t* ws_keys = nullptr;          // pass 1: nq × nranges × kprime
    const float* q_thr = nullptr;         // pass 2: per query T (exact k-th score of pass 1)
    uint32_t* cand_rows = nullptr;        // pass 2: nq × cap2
    uint32_t* cand_cnt = nullptr;         // pass 2: nq, zeroed before the launch
    uint32_t* status = nullptr;
    // IVF item mode (the list scan on the tensor cores): CTA b runs work item b of the IVF plan —
    // one chunk of one list's reordered rows against one gathered block of ≤ 128 queries probing it.
    const uint32_t* it_item_off = nullptr;    // nlist + 1: first work item of each list
    const uint32_t* it_item_list = nullptr;   // items: the list of each work item
    unsigned long long* it_next = nullptr;    // zeroed before the launch: the next item to take
    const uint32_t* it_list_cnt = nullptr;    // nlist: queries probing each list
    const uint32_t* it_offsets = nullptr;     // nlist + 1: each list's reordered row range
    const uint32_t* it_qblock_off = nullptr;  // nlist + 1: first gathered query block of each list
    const uint32_t* it_lane_qid = nullptr;    // blocks × 128: query of each lane (0xFFFFFFFF = none)
    const uint32_t* it_lane_slot = nullptr;   // blocks × 128: the query's output slot for chunk 0
    const uint32_t* row_map = nullptr;        // reordered row → original row
    uint32_t it_nlist = 0;
    uint32_t it_chunk_rows = 0;
    // Pass 2 with a device-side query count (no host round trip after pass 1): live_q[0] queries of
    // the gathered block are live; the 1-D grid's CTA b takes work item b of (query block, row
    // range), the ranges derived from the count as the host derives them (tc_ranges with sm_count).
    const uint32_t* live_q = nullptr;
    uint32_t sm_count = 0;
};
struct TcArgs {
    const CUtensorMap* tmap_q = nullptr;  // quantised queries [nq_alloc × K], box {128 B, 128 rows}
    const CUtensorMap* tmap_b = nullptr;  // quantised base [rows_alloc × K], box {128 B, 256 rows}
                                          // (qb = 2: box {128 B, 128 rows})
    TcParams p;
    uint32_t nranges = 0;
    uint32_t stages = 4;                  // base ring depth (2..4)
    bool stream_a = false;                // pass 1: query slabs staged per ring stage, not resident
    uint32_t items = 0;                   // IVF item mode: number of work items (grid), 0 = off
    uint32_t live_items = 0;              // pass 2 with p.live_q: CTAs launched (an upper bound)
    uint32_t qb = 1;                      // pass 2: query blocks per CTA (2: 128-row base tiles;
                                          // 3: one per CTA of a CTA pair, 128 of the pair's 256 rows)
};
size_t tc_smem_bytes(uint32_t nchunks, uint32_t kprime, uint32_t stages, bool fp8, bool stream_a, uint32_t qb = 1);
// Deepest base ring (4, 3 or 2 stages) that fits k′ heaps in `smem_limit`; 0 if none fits.
uint32_t tc_stages_for(uint32_t nchunks, uint32_t kprime, bool fp8, bool stream_a, size_t smem_limit);
// Pass 2 with two resident query blocks per CTA: the deepest ring (5 or 4 stages of 128-row slabs)
// that fits beside both blocks' query slabs; 0 if none (large D).
uint32_t tc_pair_stages_for(uint32_t nchunks, bool fp8, size_t smem_limit);
// Ring stages of a CTA-pair pass 2 (TcArgs::qb = 3) that fit, 0 when none does.
uint32_t tc_cta_pair_stages_for(uint32_t nchunks, bool fp8, size_t smem_limit);
cudaError_t launch_scan_tc(const TcArgs& a, bool fp8, int mode, cudaStream_t stream);

// K12: FP32-accurate candidate scan on the tensor cores (three TF32 products per K step), 16
// queries per CTA; per query and CTA the kp best keys of (s̃ + eps, row) go to ws_keys.
struct Tf32ScanArgs {
    uint32_t nq = 0;
    uint32_t nbox = 0;                 // 128-byte slabs per row (ds / 32)
    uint32_t ds = 0;                   // floats per stored row
    uint64_t rows = 0;
    uint32_t kp = 0;                   // candidates kept per query and CTA
    uint32_t cap = 0;                  // candidate buffer per query, ≥ kp + 128
    const float* queries = nullptr;    // nq × ds normalised queries (their norms are taken in-kernel)
    const float2* row_norms = nullptr; // per row {‖x‖, ‖x − tf32_head(x)‖}, rounded up
    float c_norm = 0.0f;               // C of ε: accumulation and rounding terms per unit ‖q‖‖x‖
    bool evict_first = true;           // L2 policy of the base loads (one query block: stream once)
    uint64_t* ws_keys = nullptr;       // nq × ctas × kp
    // optional, nq keys zeroed before the launch: the largest over CTAs of the smallest key of a
    // full (kp-key) list. Every row a CTA did not list has a smaller key than its list's smallest,
    // so every row outside the lists stays below it (the certificate must clear it).
    unsigned long long* floor_keys = nullptr;
    uint32_t* status = nullptr;
};
size_t tf32_smem_bytes(uint32_t stages, uint32_t cap);
uint32_t tf32_stages_for(uint32_t cap, size_t smem_limit);
// tmap_x: the FP32 base, box {32 floats, 128 rows}, 128-byte swizzle; tmap_q: the normalised
// queries (nq rows; the rows past nq read as zeros), box {32 floats, 16 rows}, 128-byte swizzle.
cudaError_t launch_scan_tf32(const CUtensorMap& tmap_x, const CUtensorMap& tmap_q, const Tf32ScanArgs& a,
                             uint32_t stages, uint32_t ctas, cudaStream_t stream);
// Per row of the base (stride ds): {‖x‖, ‖x − tf32_head(x)‖}, FP64 sums rounded up.
cudaError_t launch_tf32_row_norms(const float* base, uint64_t rows, uint32_t ds, float2* out, uint32_t sm_count,
                                  cudaStream_t stream);

// Device-side certificate fallback: compaction of the zero flags (one block), a gather of their rows
// (zeros past the count), and a scatter of re-run results back to their queries' slots.
void launch_compact_zero_flags(const uint32_t* flags, uint32_t n, uint32_t* ids, uint32_t* count, cudaStream_t s,
                               const uint32_t* live = nullptr);
void launch_gather_rows(const float* src, uint32_t ds, const uint32_t* ids, const uint32_t* count, uint32_t n,
                        float* dst, cudaStream_t s);
void launch_scatter_results(const uint64_t* fb_idx, const float* fb_sim, const uint32_t* fb_cnt, const uint32_t* ids,
                            const uint32_t* count, uint32_t n, uint32_t k, uint64_t* idx, float* sim, uint32_t* cnt,
                            cudaStream_t s);

struct RerankArgs {
    const float* base = nullptr;  // FP32 base, stride ds (with row_map: the list-ordered copy)
    uint32_t ds = 0;
    const float* queries = nullptr;  // FP32 normalised queries, stride ds
    const uint64_t* cand_idx = nullptr;  // nq × kp, sorted by upper bound
    const float* cand_sim = nullptr;     // upper bounds of the exact scores, sorted descending
    const uint32_t* cand_cnt = nullptr;
    uint32_t nq = 0, kp = 0, k = 0;
    uint64_t* idx_out = nullptr;
    float* sim_out = nullptr;
    uint32_t* cnt_out = nullptr;
    uint32_t* cert_out = nullptr;
    float* kth_out = nullptr;            // exact k-th score per query (pass-2 threshold)
    bool certify = true;                 // false when pass 1 scanned a sample of the rows
    // optional: an uncertified query appends its index to fb_ids at fb_count[0] (zeroed before)
    uint32_t* fb_ids = nullptr;
    uint32_t* fb_count = nullptr;
    // optional (IVF): candidates are list positions; base is read by position, results carry
    // row_map[position]
    const uint32_t* row_map = nullptr;
    // optional, per query: a key every row outside the candidate lists stays below (their largest
    // full-list minimum); the certificate must clear it too
    const unsigned long long* floor_keys = nullptr;
};
cudaError_t launch_rerank(const RerankArgs& a, cudaStream_t stream);
// q2_lp holds m rounded up to 128 rows (whole query blocks); the rows past m are written as zeros.
cudaError_t launch_gather_queries(const uint32_t* ids, uint32_t m, const void* q_lp, uint32_t row_bytes, void* q2_lp,
                                  const float* resid, float* resid2, const float* scale, float* scale2,
                                  const float* kth, float* thr2, cudaStream_t stream, const uint32_t* live = nullptr);
// Pass 2's exact rerank (two launches: work items of collected rows, then a merge per query).
// thr: each query's T (indexed like cnt2). vecs: the base by row, or with row_map (IVF) the
// list-ordered copy by collected position. slot_keys: m × rerank_chunks(cap2) × k keys of scratch.
uint32_t rerank_chunks(uint32_t cap2);
cudaError_t launch_rerank_collected(const float* vecs, uint32_t ds, const float* queries, const uint32_t* ids,
                                    uint32_t m, const uint32_t* rows2, const uint32_t* cnt2, uint32_t cap2, uint32_t k,
                                    const float* thr, uint64_t* slot_keys, uint64_t* idx_out, float* sim_out,
                                    uint32_t* cnt_out, uint32_t* ok_out, cudaStream_t stream, bool by_query = false,
                                    const uint32_t* live = nullptr, const uint32_t* row_map = nullptr);
cudaError_t launch_max_reduce(const float* v, uint64_t n, unsigned int* out, cudaStream_t stream);
// FP8: {min, max} row scale of each 256-row tile (tiles = rows_alloc / 256).
void launch_tile_scale(const float* row_scale, uint64_t rows, uint64_t tiles, float2* out, cudaStream_t s);

// Maximum k the fused scan kernels select in shared memory.
constexpr uint32_t kMaxFusedK = 2048;

// FP64 scores of (query, row) pairs: base rows of stride ds, queries of stride dims.
// |sim − FP64 score| of each of nq × k results (rows idx, stride k; cnt may be null = k each) into
// out, and acc = {max as double bits, sum as double, count} accumulated atomically.
void launch_score_errors(const float* base, uint64_t ds, const float* queries, uint32_t nq, uint32_t k,
                         const uint64_t* idx, const float* sim, const uint32_t* cnt, double* out,
                         unsigned long long* acc, cudaStream_t stream);
void launch_fp64_pairs(const float* base, uint64_t ds, const float* queries, uint64_t dims,
                       const uint64_t* pq, const uint64_t* pr, uint64_t n, double* out,
                       cudaStream_t stream);

}  // namespace nndex
