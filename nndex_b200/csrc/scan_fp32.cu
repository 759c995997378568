// scan_fp32.cu — K2: exact FP32 scan of the base with a fused top-k, and the cross-CTA merge.
//
// Replaces the reference's exact scoring + top-k: the CPU strategies (src/cpu.rs:256-341,
// 505-639), the wgpu shaders (src/shaders/dot_lowdim.wgsl, dot_highdim.wgsl) with their host
// top-k over a read-back score matrix (src/gpu.rs:486-785), and TopKAccumulator /
// topk_from_scores (src/topk.rs:44-210). Scores never reach HBM.
//
// Layout. The base is a row-major FP32 matrix [rows × dp] (dp = dims rounded up to 8, zero
// padded). A TMA tensor map describes it with a box of 32 floats (128 B) × TR rows and the
// 128-byte swizzle, so a tile of TR rows arrives in shared memory one 128 B column slab at a time
// (nbox = dq / 32 slabs per tile). One producer warp issues the loads into a ring of `stages`
// slabs guarded by full/empty mbarriers; NCW consumer warps compute.
//
// Consumers (scan_core.cuh): 2·NCW warps per group of up to 8 queries (16 warps at 16 queries per
// CTA), each lane a 4-row × 8-query block of FP32 partial sums in a fixed FMA order per (row, query),
// independent of the batch's composition.
//
// Fused top-k. Per query, a shared-memory buffer of `cap` 64-bit keys (common.cuh) and the
// current k-th best key `thr`. A score enters the buffer only if its key beats `thr`; when a
// buffer could overflow on the next tile, a warp radix-selects its exact k best, compacts, and
// raises `thr`. Each CTA writes its k best keys per query; merge_topk_kernel selects the global k
// best and sorts them (similarity desc, index asc).
#include <algorithm>
#include <cstdlib>

#include "common.cuh"

#include "internal.h"
#include "scan_core.cuh"
#include "select.cuh"

namespace nndex {

namespace {

NNDEX_DEVICE_INLINE uint8_t* align_1024(uint8_t* p) {
    const uint32_t a = smem_u32(p);
    return p + ((1024u - (a & 1023u)) & 1023u);
}

}  // namespace

template <int QB, int NCW, int ST>
__global__ void __launch_bounds__(ScanShape<QB, NCW>::kThreads, 1)
    scan_fp32_kernel(const __grid_constant__ CUtensorMap tmap, const float* __restrict__ queries, uint32_t nq,
                     uint32_t dq, uint64_t rows, uint32_t k, uint32_t cap,
                     const uint32_t* __restrict__ row_map, uint64_t* __restrict__ ws_keys,
                     uint32_t* __restrict__ status, const uint32_t* __restrict__ live) {
    if (live && *live == 0) return;  // a fallback launch with nothing to re-run
    using S = ScanShape<QB, NCW>;
    using Consumer = ScanConsumer<QB, NCW, ST>;
    constexpr int TR = S::kTileRows;
    constexpr uint32_t kStageBytes = S::kStageBytes;
    constexpr uint32_t kConsumers = S::kConsumers;
    constexpr uint32_t stages = ST;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = align_1024(smem_raw);
    uint8_t* stage_base = smem;
    float* q_s = reinterpret_cast<float*>(stage_base + static_cast<size_t>(stages) * kStageBytes);
    uint64_t* cand = reinterpret_cast<uint64_t*>(q_s + static_cast<size_t>(QB) * dq);
    float* xchg = reinterpret_cast<float*>(cand + static_cast<size_t>(QB) * cap);  // kConsumers × 32 × kXchg
    uint32_t* hist = reinterpret_cast<uint32_t*>(xchg + kConsumers * 32 * S::kXchg);
    uint64_t* thr = reinterpret_cast<uint64_t*>(hist + kConsumers * 256);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(thr + QB);
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(cnt + QB + (QB & 1));
    uint64_t* empty_bar = full_bar + stages;
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(empty_bar + stages);

    const uint32_t tid = threadIdx.x;
    const uint32_t warp = tid >> 5;
    const uint32_t lane = tid & 31u;
    const uint32_t G = gridDim.x;
    const uint32_t c = blockIdx.x;
    const uint32_t q0 = blockIdx.y * QB;
    const uint32_t nqg = (nq - q0) < static_cast<uint32_t>(QB) ? (nq - q0) : static_cast<uint32_t>(QB);
    // Whole tiles per CTA: only the base's last tile reads rows past the end (zero padding / TMA
    // fill), so no CTA streams rows that belong to the next one.
    const uint64_t tiles_total = (rows + TR - 1) / TR;
    const uint64_t row_begin = static_cast<uint64_t>(TR) * (tiles_total * c / G);
    const uint64_t row_end_t = static_cast<uint64_t>(TR) * (tiles_total * (c + 1) / G);
    const uint64_t row_end = row_end_t < rows ? row_end_t : rows;
    const uint32_t ntiles = static_cast<uint32_t>(row_end > row_begin ? (row_end - row_begin + TR - 1) / TR : 0);
    const uint32_t nbox = dq / 32;

    if (tid == 0) {
        for (uint32_t s = 0; s < stages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], kConsumers);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    for (uint32_t i = tid; i < static_cast<uint32_t>(QB) * dq; i += blockDim.x) {
        const uint32_t b = i / dq, d = i - b * dq;
        q_s[i] = b < nqg ? queries[static_cast<size_t>(q0 + b) * dq + d] : 0.0f;
    }
    if (tid < static_cast<uint32_t>(QB)) {
        cnt[tid] = 0;
        thr[tid] = 0ull;
    }
    __syncthreads();

    if (warp == kConsumers) {
        // ---------------- producer ----------------
        if (lane == 0) {
            tma_prefetch_desc(&tmap);
            // One query group streams each row once: evict first. Several groups read the same
            // rows at about the same time (one wave, the groups' CTAs side by side): keep them.
            const uint64_t policy = gridDim.y > 1 ? l2_policy_evict_normal() : l2_policy_evict_first();
            uint32_t it = 0;
            bool stop = false;
            for (uint32_t t = 0; t < ntiles && !stop; ++t) {
                const int32_t y = static_cast<int32_t>(row_begin + static_cast<uint64_t>(t) * TR);
                for (uint32_t bx = 0; bx < nbox; ++bx) {
                    const uint32_t s = it & (ST - 1), u = it / ST;
                    if (u > 0 && !mbar_wait_bounded(&empty_bar[s], (u - 1) & 1u, kWaitBudgetCycles)) {
                        *abort_flag = 1;
                        record_status(status, kStatusTimeout);
                        stop = true;
                        break;
                    }
                    if (*abort_flag) {
                        stop = true;
                        break;
                    }
                    mbar_arrive_expect_tx(&full_bar[s], kStageBytes);
                    tma_load_2d_hint(stage_base + static_cast<size_t>(s) * kStageBytes, &tmap, &full_bar[s],
                                     static_cast<int32_t>(bx * 32), y, policy);
                    ++it;
                }
            }
            // Drain: every issued copy has landed before the CTA may exit.
            const uint32_t used = it < stages ? it : stages;
            for (uint32_t s = 0; s < used; ++s) {
                const uint32_t uses = (it - s + stages - 1) / stages;
                if (!mbar_wait_bounded(&full_bar[s], (uses - 1) & 1u, kWaitBudgetCycles))
                    record_status(status, kStatusTimeout);
            }
        }
        return;
    }

    // ---------------- consumers ----------------
    const Consumer con(warp, lane, stage_base, q_s, dq, xchg);
    auto row_key = [&](uint64_t r) { return row_map ? row_map[r] : static_cast<uint32_t>(r); };
    float acc[4][Consumer::QW];
    uint32_t it = 0;
    for (uint32_t t = 0; t < ntiles; ++t) {
        con.accumulate(acc, nbox, it, full_bar, empty_bar, abort_flag, status);
        con.insert(acc, row_begin + static_cast<uint64_t>(t) * TR, row_end, nqg, row_key, thr, cnt, cand, cap, status);
        scan_flush<QB, NCW>(t + 1 == ntiles, nqg, k, cap, warp, lane, cnt, thr, cand, hist);
    }
    // Write this CTA's k best keys per query (0 = empty slot).
    for (uint32_t b = warp; b < nqg; b += kConsumers) {
        const uint32_t n = cnt[b] < k ? cnt[b] : k;
        uint64_t* dst = ws_keys + (static_cast<size_t>(q0 + b) * G + c) * k;
        const uint64_t* src = cand + static_cast<size_t>(b) * cap;
        for (uint32_t j = lane; j < k; j += 32) dst[j] = j < n ? src[j] : 0ull;
    }
}

// The same scan with the wide consumer (scan_core.cuh ScanConsumerWide): W consumer warps of 16
// rows × all QB (8 or 16) queries, a tile of 16·W rows arriving as 128-row TMA boxes per slab.
template <int QB, int W, int ST>
__global__ void __launch_bounds__((W + 1) * 32, 1)
    scan_fp32_wide_kernel(const __grid_constant__ CUtensorMap tmap, const float* __restrict__ queries, uint32_t nq,
                          uint32_t dq, uint64_t rows, uint32_t k, uint32_t cap,
                          const uint32_t* __restrict__ row_map, uint64_t* __restrict__ ws_keys,
                          uint32_t* __restrict__ status, const uint32_t* __restrict__ live) {
    if (live && *live == 0) return;  // a fallback launch with nothing to re-run
    using Consumer = ScanConsumerWide<QB, W, ST>;
    constexpr int TR = Consumer::kTileRows;
    constexpr uint32_t kStageBytes = Consumer::kStageBytes;
    // one box per 128 rows, or a single box of the whole tile (tensor map with box rows = TR)
    constexpr uint32_t kBoxRows = (TR % 128 == 0) ? 128 : TR;
    constexpr uint32_t kBoxes = TR / kBoxRows;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = align_1024(smem_raw);
    uint8_t* stage_base = smem;
    float* q_s = reinterpret_cast<float*>(stage_base + static_cast<size_t>(ST) * kStageBytes);
    uint64_t* cand = reinterpret_cast<uint64_t*>(q_s + static_cast<size_t>(QB) * dq);
    uint32_t* hist = reinterpret_cast<uint32_t*>(cand + static_cast<size_t>(QB) * cap);
    uint64_t* thr = reinterpret_cast<uint64_t*>(hist + W * 256);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(thr + QB);
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(cnt + QB + (QB & 1));  // mbarriers: 8-byte aligned
    uint64_t* empty_bar = full_bar + ST;
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(empty_bar + ST);

    const uint32_t tid = threadIdx.x;
    const uint32_t warp = tid >> 5;
    const uint32_t lane = tid & 31u;
    const uint32_t G = gridDim.x;
    const uint32_t c = blockIdx.x;
    const uint32_t q0 = blockIdx.y * QB;
    const uint32_t nqg = (nq - q0) < static_cast<uint32_t>(QB) ? (nq - q0) : static_cast<uint32_t>(QB);
    // Whole tiles per CTA: only the base's last tile reads rows past the end (zero padding / TMA
    // fill), so no CTA streams rows that belong to the next one.
    const uint64_t tiles_total = (rows + TR - 1) / TR;
    const uint64_t row_begin = static_cast<uint64_t>(TR) * (tiles_total * c / G);
    const uint64_t row_end_t = static_cast<uint64_t>(TR) * (tiles_total * (c + 1) / G);
    const uint64_t row_end = row_end_t < rows ? row_end_t : rows;
    const uint32_t ntiles = static_cast<uint32_t>(row_end > row_begin ? (row_end - row_begin + TR - 1) / TR : 0);
    const uint32_t nbox = dq / 32;

    if (tid == 0) {
        for (uint32_t s = 0; s < ST; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], W * 32);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    // queries slab-major (ScanConsumerWide::q_slab_index)
    for (uint32_t i = tid; i < static_cast<uint32_t>(QB) * dq; i += blockDim.x) {
        const uint32_t b = i / dq, d = i - b * dq;
        q_s[Consumer::q_slab_index(b, d)] = b < nqg ? queries[static_cast<size_t>(q0 + b) * dq + d] : 0.0f;
    }
    if (tid < static_cast<uint32_t>(QB)) {
        cnt[tid] = 0;
        thr[tid] = 0ull;
    }
    __syncthreads();

    if (warp == W) {
        // ---------------- producer ----------------
        if (lane == 0) {
            tma_prefetch_desc(&tmap);
            // One query group streams each row once: evict first. Several groups read the same
            // rows at about the same time (one wave, the groups' CTAs side by side): keep them.
            const uint64_t policy = gridDim.y > 1 ? l2_policy_evict_normal() : l2_policy_evict_first();
            uint32_t it = 0;
            bool stop = false;
            for (uint32_t t = 0; t < ntiles && !stop; ++t) {
                const int32_t y = static_cast<int32_t>(row_begin + static_cast<uint64_t>(t) * TR);
                for (uint32_t bx = 0; bx < nbox; ++bx) {
                    const uint32_t s = it % ST, u = it / ST;
                    if (u > 0 && !mbar_wait_bounded_suspend(&empty_bar[s], (u - 1) & 1u, kWaitBudgetCycles, 20000)) {
                        *abort_flag = 1;
                        record_status(status, kStatusTimeout);
                        stop = true;
                        break;
                    }
                    if (*abort_flag) {
                        stop = true;
                        break;
                    }
                    mbar_arrive_expect_tx(&full_bar[s], kStageBytes);
#pragma unroll
                    for (uint32_t h = 0; h < kBoxes; ++h)
                        tma_load_2d_hint(stage_base + static_cast<size_t>(s) * kStageBytes + h * kBoxRows * 128, &tmap,
                                         &full_bar[s], static_cast<int32_t>(bx * 32),
                                         y + static_cast<int32_t>(h * kBoxRows), policy);
                    ++it;
                }
            }
            // Drain: every issued copy has landed before the CTA may exit.
            const uint32_t used = it < ST ? it : ST;
            for (uint32_t s = 0; s < used; ++s) {
                const uint32_t uses = (it - s + ST - 1) / ST;
                if (!mbar_wait_bounded(&full_bar[s], (uses - 1) & 1u, kWaitBudgetCycles))
                    record_status(status, kStatusTimeout);
            }
        }
        return;
    }

    // ---------------- consumers ----------------
    const Consumer con(warp, lane, stage_base, q_s);
    auto row_key = [&](uint64_t r) { return row_map ? row_map[r] : static_cast<uint32_t>(r); };
    float acc[4][QB];
    RingPos<ST> pos;
    for (uint32_t t = 0; t < ntiles; ++t) {
        con.accumulate(acc, nbox, pos, full_bar, empty_bar, abort_flag, status);
        con.insert(acc, row_begin + static_cast<uint64_t>(t) * TR, row_end, nqg, row_key, thr, cnt, cand, cap, status);
        scan_flush_g<QB, W, TR>(t + 1 == ntiles, nqg, k, cap, warp, lane, cnt, thr, cand, hist);
    }
    for (uint32_t b = warp; b < nqg; b += W) {
        const uint32_t n = cnt[b] < k ? cnt[b] : k;
        uint64_t* dst = ws_keys + (static_cast<size_t>(q0 + b) * G + c) * k;
        const uint64_t* src = cand + static_cast<size_t>(b) * cap;
        for (uint32_t j = lane; j < k; j += 32) dst[j] = j < n ? src[j] : 0ull;
    }
}

// ------------------------------------------------------------------------------------------
// Cross-CTA merge: the k best of a query's candidate keys (one list of k per scan CTA), written
// sorted (similarity desc, index asc), the unused slots padded with (0, 0.0f)
// (src/python_bindings.rs:477-483). With `parts` > 1 the lists are split over that many blocks
// per query: each selects the exact k best of its share into part_keys, and the block that
// finishes last (a per-query counter) merges the parts·k survivors — the same result, with the
// selection work spread over parts·nq blocks instead of nq.
// ------------------------------------------------------------------------------------------
namespace {

// The k best of keys[0..n) (0 = empty slot) into the outputs of query q, sorted.
NNDEX_DEVICE_INLINE void merge_final(const uint64_t* keys, uint64_t n, uint32_t k, uint32_t q, uint32_t out_stride,
                                     uint64_t* idx_out, float* sim_out, uint32_t* count_out, BlockSelectScratch& s,
                                     uint64_t* sorted) {
    if (threadIdx.x == 0) s.count = 0;
    __syncthreads();
    uint32_t local = 0;
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) local += keys[i] != 0ull;
    local = __reduce_add_sync(0xffffffffu, local);
    if ((threadIdx.x & 31u) == 0) atomicAdd(&s.count, local);
    __syncthreads();
    const uint32_t nvalid = s.count;
    const uint32_t kk = nvalid < k ? nvalid : k;
    __syncthreads();
    uint32_t p2 = 1;
    while (p2 < kk) p2 <<= 1;
    if (kk > 0) {
        uint64_t kth = 1ull;
        if (n > kk) kth = block_radix_kth(keys, n, kk, s);
        if (threadIdx.x == 0) s.count = 0;
        __syncthreads();
        for (uint64_t i0 = 0; i0 < n; i0 += blockDim.x) {
            const uint64_t i = i0 + threadIdx.x;
            const uint64_t key = i < n ? keys[i] : 0ull;
            const bool take = key != 0ull && key >= kth;
            const uint32_t pos = warp_append(&s.count, take);
            if (take && pos < kk) sorted[pos] = key;
        }
        __syncthreads();
        // Exactly kk keys reach the k-th (keys are distinct); should fewer arrive, the slots they
        // did not fill are cleared rather than read.
        const uint32_t got = s.count < kk ? s.count : kk;
        for (uint32_t i = got + threadIdx.x; i < p2; i += blockDim.x) sorted[i] = 0ull;
        __syncthreads();
        block_bitonic_sort_desc(sorted, p2);
        __syncthreads();
        if (threadIdx.x == 0) s.count = got;
        __syncthreads();
    }
    const uint32_t out_n = kk > 0 ? s.count : 0u;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < out_stride; j += blockDim.x) {
        uint64_t idx = 0;
        float sim = 0.0f;
        if (j < out_n) {
            idx = key_row(sorted[j]);
            sim = key_score(sorted[j]);
        }
        idx_out[static_cast<size_t>(q) * out_stride + j] = idx;
        sim_out[static_cast<size_t>(q) * out_stride + j] = sim;
    }
    if (threadIdx.x == 0 && count_out) count_out[q] = out_n;
}

}  // namespace

// grid (parts, nq); dynamic shared memory: p2(k) keys for the sort, plus parts·k keys when
// parts > 1 (the survivors, staged for the final merge).
__global__ void __launch_bounds__(512) merge_topk_kernel(const uint64_t* __restrict__ ws_keys, uint64_t per_query,
                                                         uint32_t k, uint32_t out_stride,
                                                         uint64_t* __restrict__ idx_out,
                                                         float* __restrict__ sim_out,
                                                         uint32_t* __restrict__ count_out, uint32_t parts,
                                                         uint64_t* __restrict__ part_keys,
                                                         uint32_t* __restrict__ part_done,
                                                         const uint32_t* __restrict__ live,
                                                         const uint32_t* __restrict__ out_rows) {
    if (live && blockIdx.y >= *live) return;  // a fallback merge: only the queries re-run
    __shared__ BlockSelectScratch s;
    __shared__ uint32_t last;
    extern __shared__ uint64_t smem_keys[];
    const uint32_t q = blockIdx.y;
    const uint64_t* keys = ws_keys + static_cast<size_t>(q) * per_query;
    uint32_t p2 = 1;
    while (p2 < k) p2 <<= 1;
    const uint32_t oq = out_rows ? out_rows[q] : q;  // the output row of this query's results
    if (parts == 1) {
        merge_final(keys, per_query, k, oq, out_stride, idx_out, sim_out, count_out, s, smem_keys);
        return;
    }
    // This block's share of the query's keys.
    const uint64_t i0 = per_query * blockIdx.x / parts, i1 = per_query * (blockIdx.x + 1) / parts;
    const uint64_t n = i1 - i0;
    const uint64_t* src = keys + i0;
    uint64_t* dst = part_keys + (static_cast<size_t>(q) * parts + blockIdx.x) * k;
    {
        uint64_t kth = 0ull;
        if (n > k) kth = block_radix_kth(src, n, k, s);
        if (threadIdx.x == 0) s.count = 0;
        __syncthreads();
        // Non-empty keys >= kth: exactly k of them when the share holds at least k (keys are
        // distinct); all of them otherwise (kth is then an empty slot, 0). The rest of the part is
        // padded with 0.
        for (uint64_t i0 = 0; i0 < n; i0 += blockDim.x) {
            const uint64_t i = i0 + threadIdx.x;
            const uint64_t key = i < n ? src[i] : 0ull;
            const bool take = key != 0ull && key >= kth;
            const uint32_t pos = warp_append(&s.count, take);
            if (take && pos < k) dst[pos] = key;
        }
        __syncthreads();
    }
    for (uint32_t j = s.count + threadIdx.x; j < k; j += blockDim.x) dst[j] = 0ull;
    // Publish the part; the last block of this query merges them.
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&part_done[q], 1u) == parts - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the parts' non-empty keys, packed (their order does not matter to the selection)
    uint64_t* staged = smem_keys + p2;
    const uint64_t* all = part_keys + static_cast<size_t>(q) * parts * k;
    if (threadIdx.x == 0) s.count = 0;
    __syncthreads();
    for (uint32_t i0 = 0; i0 < parts * k; i0 += blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        const uint64_t key = i < parts * k ? __ldcg(all + i) : 0ull;
        const uint32_t pos = warp_append(&s.count, key != 0ull);
        if (key != 0ull) staged[pos] = key;
    }
    __syncthreads();
    const uint32_t m = s.count;
    __syncthreads();
    merge_final(staged, m, k, oq, out_stride, idx_out, sim_out, count_out, s, smem_keys);
    if (threadIdx.x == 0) part_done[q] = 0;  // ready for the next launch
}

// ------------------------------------------------------------------------------------------
// FP64 oracle scores of (query, row) pairs — the score-error report.
// ------------------------------------------------------------------------------------------
// base rows have stride `ds`; queries have stride `dims`; both are read over `dims` values.
__global__ void fp64_pairs_kernel(const float* __restrict__ base, uint64_t ds, const float* __restrict__ queries,
                                  uint64_t dims, const uint64_t* __restrict__ pq, const uint64_t* __restrict__ pr,
                                  uint64_t n, double* __restrict__ out) {
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (warp >= n) return;
    const float* x = base + pr[warp] * ds;
    const float* qv = queries + pq[warp] * dims;
    double acc = 0.0;
    for (uint64_t d = lane; d < dims; d += 32) acc = fma(static_cast<double>(x[d]), static_cast<double>(qv[d]), acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[warp] = acc;
}

// Score error of each result: one warp per (query, slot) pair, |returned score − FP64 score of the
// stored row with the normalised query|; slots past the query's count get 0. acc = {max (as the
// bits of a non-negative double, which order like the values), sum, count}.
__global__ void score_error_kernel(const float* __restrict__ base, uint64_t ds, const float* __restrict__ queries,
                                   uint32_t nq, uint32_t k, const uint64_t* __restrict__ idx,
                                   const float* __restrict__ sim, const uint32_t* __restrict__ cnt,
                                   double* __restrict__ out, unsigned long long* __restrict__ acc) {
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (warp >= static_cast<uint64_t>(nq) * k) return;
    const uint32_t q = static_cast<uint32_t>(warp / k), j = static_cast<uint32_t>(warp % k);
    const uint32_t n = cnt ? cnt[q] : k;
    if (j >= n) {
        if (lane == 0) out[warp] = 0.0;
        return;
    }
    const float* x = base + idx[warp] * ds;
    const float* qv = queries + static_cast<uint64_t>(q) * ds;
    double a = 0.0;
    for (uint64_t d = lane; d < ds; d += 32) a = fma(static_cast<double>(x[d]), static_cast<double>(qv[d]), a);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) {
        const double e = fabs(static_cast<double>(sim[warp]) - a);
        out[warp] = e;
        atomicMax(&acc[0], static_cast<unsigned long long>(__double_as_longlong(e)));
        atomicAdd(reinterpret_cast<double*>(&acc[1]), e);
        atomicAdd(&acc[2], 1ull);
    }
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
namespace {
constexpr int kNcw = 4;
constexpr int kTileRows = kNcw * 32;

size_t scan_smem_bytes(uint32_t qb, uint32_t dq, uint32_t cap, uint32_t stages) {
    const size_t consumers = scan_consumers(qb, kNcw);
    size_t b = 1024;  // alignment slack
    b += static_cast<size_t>(stages) * kTileRows * 128;
    b += static_cast<size_t>(qb) * dq * 4;
    b += static_cast<size_t>(qb) * cap * 8;
    b += consumers * 32 * scan_xchg_per_lane(qb) * 4;  // partner exchange
    b += consumers * 256 * 4;
    b += qb * 8 + (qb + (qb & 1)) * 4;
    b += static_cast<size_t>(stages) * 16 + 16;
    return b;
}

template <int QB, int ST>
cudaError_t launch_qb_st(const ScanArgs& a, const ScanPlan& p, cudaStream_t stream) {
    auto kern = scan_fp32_kernel<QB, kNcw, ST>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(p.smem_bytes));
    if (e != cudaSuccess) return e;
    dim3 grid(p.ctas_per_group, p.groups);
    kern<<<grid, ScanShape<QB, kNcw>::kThreads, p.smem_bytes, stream>>>(*a.tmap, a.queries, a.nq, a.dq, a.rows, a.k, p.cap,
                                                              a.row_map, a.ws_keys, a.status, a.live);
    count_launch();
    return cudaGetLastError();
}

template <int QB>
cudaError_t launch_qb(const ScanArgs& a, const ScanPlan& p, cudaStream_t stream) {
    return p.stages >= 4 ? launch_qb_st<QB, 4>(a, p, stream) : launch_qb_st<QB, 2>(a, p, stream);
}

size_t wide_smem_bytes(uint32_t qb, uint32_t w, uint32_t dq, uint32_t cap, uint32_t stages) {
    size_t b = 1024;
    b += static_cast<size_t>(stages) * w * 16 * 128;
    b += static_cast<size_t>(qb) * dq * 4;
    b += static_cast<size_t>(qb) * cap * 8;
    b += static_cast<size_t>(w) * 256 * 4;
    b += qb * 8 + (qb + (qb & 1)) * 4;
    b += static_cast<size_t>(stages) * 16 + 16;
    return b;
}

template <int QB, int W, int ST>
cudaError_t launch_wide_st(const ScanArgs& a, const ScanPlan& p, cudaStream_t stream) {
    auto kern = scan_fp32_wide_kernel<QB, W, ST>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(p.smem_bytes));
    if (e != cudaSuccess) return e;
    // tiles of 16·W rows: 128-row boxes, or one box of the tile (a tensor map of that box height)
    const CUtensorMap* tm = (16 * W) % 128 == 0 ? a.tmap : (W == 7 ? a.tmap_112 : a.tmap_tile);
    if (!tm) return cudaErrorInvalidValue;
    dim3 grid(p.ctas_per_group, p.groups);
    kern<<<grid, (W + 1) * 32, p.smem_bytes, stream>>>(*tm, a.queries, a.nq, a.dq, a.rows, a.k, p.cap, a.row_map,
                                                       a.ws_keys, a.status, a.live);
    count_launch();
    return cudaGetLastError();
}

template <int QB>
cudaError_t launch_wide(const ScanArgs& a, const ScanPlan& p, cudaStream_t stream) {
    if (p.wide == 11) {
        switch (p.stages) {
            case 2: return launch_wide_st<QB, 11, 2>(a, p, stream);
            case 3: return launch_wide_st<QB, 11, 3>(a, p, stream);
            case 5: return launch_wide_st<QB, 11, 5>(a, p, stream);
            default: return launch_wide_st<QB, 11, 4>(a, p, stream);
        }
    }
    if (p.wide == 7) {
        switch (p.stages) {
            case 2: return launch_wide_st<QB, 7, 2>(a, p, stream);
            case 4: return launch_wide_st<QB, 7, 4>(a, p, stream);
            case 6: return launch_wide_st<QB, 7, 6>(a, p, stream);
            default: return launch_wide_st<QB, 7, 8>(a, p, stream);
        }
    }
    if (p.wide == 16) {
        switch (p.stages) {
            case 2: return launch_wide_st<QB, 16, 2>(a, p, stream);
            case 3: return launch_wide_st<QB, 16, 3>(a, p, stream);
            default: return launch_wide_st<QB, 16, 4>(a, p, stream);
        }
    }
    switch (p.stages) {
        case 2: return launch_wide_st<QB, 8, 2>(a, p, stream);
        case 3: return launch_wide_st<QB, 8, 3>(a, p, stream);
        case 6: return launch_wide_st<QB, 8, 6>(a, p, stream);
        case 8: return launch_wide_st<QB, 8, 8>(a, p, stream);
        default: return launch_wide_st<QB, 8, 4>(a, p, stream);
    }
}
}  // namespace

// Tile-shape overrides for the autotuner and for measurement sweeps (0 = default):
//   NNDEX_SCAN_STAGES   ring depth (2 or 4)        NNDEX_SCAN_QB   max queries per CTA (1..16)
//   NNDEX_SCAN_CTAS     CTAs per query group      NNDEX_SCAN_CAP  candidate slots beyond k
//   NNDEX_SCAN_WIDE     wide consumer warps at 1..16 queries per CTA: 7, 8, 11 or 16 (default 16
//                       up to 8 queries, 11 at 16); 1 = the 4-row × 8-query consumer instead
static uint32_t env_u32(const char* name) {
    const char* v = getenv(name);
    return v ? static_cast<uint32_t>(strtoul(v, nullptr, 10)) : 0u;
}

bool plan_scan_fp32(uint32_t nq, uint32_t dq, uint32_t k, uint64_t rows, int sm_count, size_t smem_limit,
                    ScanPlan& plan) {
    if (k == 0 || k > kMaxFusedK || nq == 0) return false;
    static const uint32_t o_stages = env_u32("NNDEX_SCAN_STAGES"), o_qb = env_u32("NNDEX_SCAN_QB"),
                          o_ctas = env_u32("NNDEX_SCAN_CTAS"), o_cap = env_u32("NNDEX_SCAN_CAP");
    uint32_t qb = nq <= 1 ? 1 : nq <= 2 ? 2 : nq <= 4 ? 4 : nq <= 8 ? 8 : 16;
    if (o_qb) while (qb > 1 && qb > o_qb) qb >>= 1;
    const uint32_t extra = o_cap ? (o_cap > kTileRows ? o_cap : kTileRows + 32) : 2 * kTileRows;
    const uint32_t cap = ((k + extra) + 31) / 32 * 32;
    const uint32_t max_stages = (o_stages && o_stages < 4) ? 2 : 4;
    for (;;) {
        uint32_t stages = max_stages;
        while (stages >= 2 && scan_smem_bytes(qb, dq, cap, stages) > smem_limit) stages >>= 1;
        if (stages >= 2) {
            plan.qb = qb;
            plan.cap = cap;
            plan.stages = stages;
            plan.smem_bytes = scan_smem_bytes(qb, dq, cap, stages);
            break;
        }
        if (qb == 1) return false;
        qb >>= 1;
    }
    // 8 or 16 queries per CTA: the wide consumer (16 rows × all queries per warp) when it fits.
    static const uint32_t o_wide = env_u32("NNDEX_SCAN_WIDE");
    plan.wide = 0;
    if (o_wide != 1) {
        // 16 consumer warps at 8 queries (96 registers, 4 warps per scheduler); 11 at 16 queries (3
        // per scheduler at up to 168 registers: the 64 accumulators need more than the 96 registers
        // that 17 warps leave)
        const uint32_t w = o_wide ? (o_wide == 16 || o_wide == 11 || o_wide == 7 ? o_wide : 8)
                                  : (plan.qb <= 8 ? 16 : 11);
        const uint32_t tr = 16 * w;
        const uint32_t wcap = ((k + (o_cap ? (o_cap > tr ? o_cap : tr + 32) : 2 * tr)) + 31) / 32 * 32;
        // ring depths with a kernel instance: 16 warps {4, 3, 2}, 8 warps {6, 4, 3, 2}
        static const uint32_t kDepth16[] = {4, 3, 2, 0}, kDepth11[] = {5, 4, 3, 2, 0},
                              kDepth8[] = {8, 6, 4, 3, 2, 0}, kDepth7[] = {8, 6, 4, 2, 0};
        const uint32_t* depths = w == 16 ? kDepth16 : w == 11 ? kDepth11 : w == 7 ? kDepth7 : kDepth8;
        uint32_t st = 0;
        for (const uint32_t* d = depths; *d; ++d) {
            if (o_stages && *d > o_stages) continue;
            if (wide_smem_bytes(plan.qb, w, dq, wcap, *d) <= smem_limit) {
                st = *d;
                break;
            }
        }
        if (st >= 2) {
            plan.wide = w;
            plan.cap = wcap;
            plan.stages = st;
            plan.smem_bytes = wide_smem_bytes(plan.qb, w, dq, wcap, st);
        }
    }
    plan.groups = (nq + plan.qb - 1) / plan.qb;
    // CTAs per query group (each taking 1/per of the rows): a CTA fills an SM, so the launch takes
    // ceil(groups × per / SMs) rounds of 1/per of the base. The rule fills the SMs once (per = SMs /
    // groups); where that leaves a last round part-empty by more than 5 %, per minimises rounds / per
    // over at most 8 rounds, with at least 2,048 rows per CTA (256 groups of one CTA, at 4,096
    // queries, took 2 rounds where 1.73 was the ideal; 4 CTAs per group take 1.75).
    const uint64_t sms = static_cast<uint64_t>(sm_count > 0 ? sm_count : 1);
    const uint64_t base_per = std::max<uint64_t>(1, sms / plan.groups);
    const uint64_t base_rounds = (plan.groups * base_per + sms - 1) / sms;
    uint64_t per_cap = std::min<uint64_t>(8 * sms / plan.groups, rows / 2048);
    per_cap = std::min<uint64_t>(std::max<uint64_t>(per_cap, base_per), 1024);
    uint64_t best = base_per, best_rounds = base_rounds;
    for (uint64_t c = 1; c <= per_cap; ++c) {
        const uint64_t r = (plan.groups * c + sms - 1) / sms;
        if (r * best < best_rounds * c) {  // r / c < best_rounds / best
            best = c;
            best_rounds = r;
        }
    }
    // keep the rule unless the split is ≥ 5 % faster: best_rounds / best ≤ 0.95 · base_rounds / base_per
    uint32_t per = static_cast<uint32_t>(base_per);
    if (best_rounds * base_per * 100 <= base_rounds * best * 95) per = static_cast<uint32_t>(best);
    if (o_ctas) per = o_ctas;
    plan.ctas_per_group = per;
    return true;
}

cudaError_t launch_scan_fp32(const ScanArgs& a, const ScanPlan& p, cudaStream_t stream) {
    if (p.wide) {
        switch (p.qb) {
            case 1: return launch_wide<1>(a, p, stream);
            case 2: return launch_wide<2>(a, p, stream);
            case 4: return launch_wide<4>(a, p, stream);
            case 8: return launch_wide<8>(a, p, stream);
            default: return launch_wide<16>(a, p, stream);
        }
    }
    switch (p.qb) {
        case 1: return launch_qb<1>(a, p, stream);
        case 2: return launch_qb<2>(a, p, stream);
        case 4: return launch_qb<4>(a, p, stream);
        case 8: return launch_qb<8>(a, p, stream);
        case 16: return launch_qb<16>(a, p, stream);
        default: return cudaErrorInvalidValue;
    }
}

uint32_t merge_parts(uint64_t per_query, uint32_t k, uint32_t nq) {
    const uint64_t lists = k ? per_query / k : 0;
    uint64_t parts = lists < 16 ? lists : 16;
    while (parts > 1 && parts * k > 4096) --parts;  // survivors staged in shared memory
    // Splitting a query's lists over blocks only helps while the queries alone leave SMs idle: about
    // 1,024 blocks in all. (At 4,096 queries, 16 parts made 65,536 blocks, each a full block radix
    // select over about 74 keys: 2.0 ms, against 0.04 ms for the rerank that follows.)
    const uint64_t by_blocks = nq ? (1024 + nq - 1) / nq : 1;
    if (parts > by_blocks) parts = by_blocks;
    return parts < 1 ? 1u : static_cast<uint32_t>(parts);
}

cudaError_t launch_merge_topk(const MergeArgs& a, cudaStream_t stream) {
    uint32_t p2 = 1;
    while (p2 < a.k) p2 <<= 1;
    const uint32_t parts = (a.part_keys && a.part_done) ? merge_parts(a.per_query, a.k, a.nq) : 1u;
    const size_t smem = (p2 + (parts > 1 ? static_cast<size_t>(parts) * a.k : 0)) * sizeof(uint64_t);
    if (smem > 40 * 1024) {  // with the static scratch, above the default 48 KB per block
        cudaError_t e = cudaFuncSetAttribute(merge_topk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    merge_topk_kernel<<<dim3(parts, a.nq), 512, smem, stream>>>(a.ws_keys, a.per_query, a.k, a.out_stride, a.idx_out,
                                                                a.sim_out, a.count_out, parts, a.part_keys,
                                                                a.part_done, a.live, a.out_rows);
    count_launch();
    return cudaGetLastError();
}

void launch_score_errors(const float* base, uint64_t ds, const float* queries, uint32_t nq, uint32_t k,
                         const uint64_t* idx, const float* sim, const uint32_t* cnt, double* out,
                         unsigned long long* acc, cudaStream_t stream) {
    const uint64_t n = static_cast<uint64_t>(nq) * k;
    if (n == 0) return;
    const uint64_t blocks = (n * 32 + 255) / 256;
    score_error_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(base, ds, queries, nq, k, idx, sim, cnt, out,
                                                                        acc);
    count_launch();
}

void launch_fp64_pairs(const float* base, uint64_t ds, const float* queries, uint64_t dims, const uint64_t* pq,
                       const uint64_t* pr, uint64_t n, double* out, cudaStream_t stream) {
    if (n == 0) return;
    const uint64_t blocks = (n * 32 + 255) / 256;
    fp64_pairs_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(base, ds, queries, dims, pq, pr, n, out);
    count_launch();
}

}  // namespace nndex
