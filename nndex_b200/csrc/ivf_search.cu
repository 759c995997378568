// ivf_search.cu — K8/K9: IVF probe and the ragged list scan with exact FP32 rerank.
//
// Replaces candidate_clusters(_batch) (src/approx.rs:159-300) and search_approx /
// search_batch_approx (src/cpu.rs:425-502). A batch runs as four launches and no host round trip:
//   1. probe: per query, dot_small against every centroid (FP64 in index order, f32 result — the
//      reference's value) and the nprobe best clusters (score desc, lower index on ties).
//   2. plan (one block): the (list, query) pairs grouped by list, each list cut into chunks of at
//      most kChunkRows rows, and work items (list chunk × group of up to QB queries probing it),
//      with every (query, list chunk) owning one output slot of k keys.
//   3. scan: persistent CTAs take work items from a global counter. A list chunk streams through
//      shared memory by TMA once per item while up to QB queries are scored against it with the
//      FP32 scan's exact FMA order (so an IVF score is bit-identical to the exact path's score of
//      the same row), and each query's best k keys of the chunk go to its slot.
//   4. merge: per query, the best k of its slots, sorted (similarity desc, index asc).
// Lists probed by many queries are read once per group of QB queries: the list scan is bounded by
// the union of probed rows, not by the sum over queries.
#include <algorithm>

#include "common.cuh"
#include "index.h"
#include "internal.h"
#include "ivf.h"
#include "scan_core.cuh"
#include "select.cuh"

namespace nndex {

namespace {
constexpr uint32_t kChunkRows = 4096;   // rows per list chunk (work-item granularity)
constexpr int kNcw = 4;                 // consumer warps per half (as the FP32 scan)
constexpr int kTileRows = kNcw * 32;    // 128 rows per tile
constexpr int kStages = 4;
constexpr uint32_t kStageBytes = kTileRows * 128;

NNDEX_DEVICE_INLINE uint8_t* align_1024(uint8_t* p) {
    const uint32_t a = smem_u32(p);
    return p + ((1024u - (a & 1023u)) & 1023u);
}

NNDEX_DEVICE_INLINE float fold_zero(float f) { return f == 0.0f ? 0.0f : f; }

// In-place exclusive scan of v[0..n) by one block; v[n] = total.
NNDEX_DEVICE_INLINE void block_exclusive_scan(uint32_t* v, uint32_t n, uint32_t* part) {
    const uint32_t t = threadIdx.x, nt = blockDim.x;
    const uint32_t per = (n + nt - 1) / nt;
    const uint32_t b = t * per, e = (b + per) < n ? (b + per) : n;
    uint32_t s = 0;
    for (uint32_t i = b; i < e; ++i) s += v[i];
    part[t] = s;
    __syncthreads();
    for (uint32_t o = 1; o < nt; o <<= 1) {
        const uint32_t x = t >= o ? part[t - o] : 0u;
        __syncthreads();
        part[t] += x;
        __syncthreads();
    }
    uint32_t run = part[t] - s;
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t x = v[i];
        v[i] = run;
        run += x;
    }
    if (t == nt - 1) v[n] = part[nt - 1];
    __syncthreads();
}
}  // namespace

// ------------------------------------------------------------------------------------------
// 1. Probe: one block per query.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    ivf_probe_kernel(const float* __restrict__ queries, uint32_t ds, uint32_t dp, const float* __restrict__ cent_t,
                     uint64_t ct_stride, uint32_t nlist, uint32_t np, uint32_t* __restrict__ probes) {
    extern __shared__ uint8_t smem_raw[];
    float* qs = reinterpret_cast<float*>(smem_raw);
    uint64_t* keys = reinterpret_cast<uint64_t*>(qs + ds);
    __shared__ BlockSelectScratch sel;
    const uint32_t q = blockIdx.x;
    for (uint32_t d = threadIdx.x; d < ds; d += blockDim.x) qs[d] = queries[static_cast<uint64_t>(q) * ds + d];
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < nlist; c += blockDim.x) {
        double s = 0.0;
        for (uint32_t d = 0; d < dp; ++d)
            s = fma(static_cast<double>(cent_t[static_cast<uint64_t>(d) * ct_stride + c]), static_cast<double>(qs[d]), s);
        keys[c] = make_key(fold_zero(__double2float_rn(s)), c);
    }
    __syncthreads();
    uint64_t kth = 0;
    if (np < nlist) kth = block_radix_kth(keys, nlist, np, sel);
    if (threadIdx.x == 0) sel.count = 0;
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < nlist; c += blockDim.x) {
        const uint64_t key = keys[c];
        if (key >= kth) {
            const uint32_t pos = atomicAdd(&sel.count, 1u);
            if (pos < np) probes[static_cast<uint64_t>(q) * np + pos] = key_row(key);
        }
    }
}

// ------------------------------------------------------------------------------------------
// 2. Plan: one block.
//    counters[0] work-item counter (the scan's), [1] items, [2] slots; summed over the sub-batches of
//    a search: [3] Σ rows probed per query, [4] rows streamed by the scan, [5] rows of probed lists.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024)
    ivf_plan_kernel(const uint32_t* __restrict__ probes, uint32_t nq, uint32_t np, uint32_t nlist,
                    const uint32_t* __restrict__ offsets, uint32_t qb, uint32_t* __restrict__ list_cnt,
                    uint32_t* __restrict__ list_fill, uint32_t* __restrict__ list_qoff, uint32_t* __restrict__ item_off,
                    uint32_t* __restrict__ list_q, uint32_t* __restrict__ list_slot, uint32_t* __restrict__ q_slot_off,
                    unsigned long long* __restrict__ counters) {
    __shared__ uint32_t part[1024];
    __shared__ unsigned long long probed;
    if (threadIdx.x == 0) probed = 0;
    __syncthreads();
    auto chunks = [&](uint32_t l) {
        const uint32_t len = offsets[l + 1] - offsets[l];
        return (len + kChunkRows - 1) / kChunkRows;
    };
    unsigned long long my_rows = 0;
    for (uint32_t q = threadIdx.x; q < nq; q += blockDim.x) {
        uint32_t slots = 0;
        for (uint32_t j = 0; j < np; ++j) {
            const uint32_t l = probes[static_cast<uint64_t>(q) * np + j];
            atomicAdd(&list_cnt[l], 1u);
            slots += chunks(l);
            my_rows += offsets[l + 1] - offsets[l];
        }
        q_slot_off[q] = slots;
    }
    atomicAdd(&probed, my_rows);
    __syncthreads();
    unsigned long long my_stream = 0, my_union = 0;
    for (uint32_t l = threadIdx.x; l < nlist; l += blockDim.x) {
        const uint32_t c = list_cnt[l];
        const uint32_t groups = (c + qb - 1) / qb;
        item_off[l] = chunks(l) * groups;
        list_qoff[l] = c;
        const uint32_t len = offsets[l + 1] - offsets[l];
        my_stream += static_cast<unsigned long long>(len) * groups;
        my_union += c ? len : 0u;
    }
    atomicAdd(&counters[4], my_stream);
    atomicAdd(&counters[5], my_union);
    __syncthreads();
    block_exclusive_scan(list_qoff, nlist, part);
    block_exclusive_scan(item_off, nlist, part);
    block_exclusive_scan(q_slot_off, nq, part);
    for (uint32_t q = threadIdx.x; q < nq; q += blockDim.x) {
        uint32_t rel = q_slot_off[q];
        for (uint32_t j = 0; j < np; ++j) {
            const uint32_t l = probes[static_cast<uint64_t>(q) * np + j];
            const uint32_t pos = list_qoff[l] + atomicAdd(&list_fill[l], 1u);
            list_q[pos] = q;
            list_slot[pos] = rel;
            rel += chunks(l);
        }
    }
    if (threadIdx.x == 0) {
        counters[0] = 0;
        counters[1] = item_off[nlist];
        counters[2] = q_slot_off[nq];
        counters[3] += probed;  // zeroed once per search: Σ over sub-batches
    }
}

// ------------------------------------------------------------------------------------------
// 3. Ragged list scan (persistent). Producer warp: TMA of 128-row × 128-byte slabs of the
//    reordered rows. 2·kNcw consumer warps: the FP32 scan's mapping and FMA order.
// ------------------------------------------------------------------------------------------
struct IvfScanArgs {
    uint32_t dq = 0;             // row stride (floats), multiple of 32
    uint32_t k = 0;
    uint32_t cap = 0;            // candidate buffer per query
    uint32_t nlist = 0;
    const float* queries = nullptr;       // normalised, stride dq
    const uint32_t* offsets = nullptr;    // nlist + 1
    const uint32_t* row_map = nullptr;    // reordered position → original row
    const uint32_t* list_cnt = nullptr;
    const uint32_t* list_qoff = nullptr;
    const uint32_t* item_off = nullptr;
    const uint32_t* list_q = nullptr;
    const uint32_t* list_slot = nullptr;
    unsigned long long* counters = nullptr;
    uint64_t* ws = nullptr;      // slots × k keys
    uint32_t* status = nullptr;
};

template <int QB>
__global__ void __launch_bounds__(ScanShape<QB, kNcw>::kThreads, 1)
    ivf_scan_kernel(const __grid_constant__ CUtensorMap tmap, const IvfScanArgs a) {
    using S = ScanShape<QB, kNcw>;
    using Consumer = ScanConsumer<QB, kNcw, kStages>;
    constexpr uint32_t kConsumers = S::kConsumers;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* stage_base = align_1024(smem_raw);
    const uint32_t dq = a.dq, cap = a.cap, k = a.k;
    float* q_s = reinterpret_cast<float*>(stage_base + static_cast<size_t>(kStages) * kStageBytes);
    uint64_t* cand = reinterpret_cast<uint64_t*>(q_s + static_cast<size_t>(QB) * dq);
    float* xchg = reinterpret_cast<float*>(cand + static_cast<size_t>(QB) * cap);
    uint32_t* hist = reinterpret_cast<uint32_t*>(xchg + kConsumers * 32 * S::kXchg);
    uint64_t* thr = reinterpret_cast<uint64_t*>(hist + kConsumers * 256);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(thr + QB);
    uint32_t* qid = cnt + QB;
    uint32_t* slot = qid + QB;
    uint64_t* item = reinterpret_cast<uint64_t*>(slot + QB + (QB & 1));  // [0] row_begin, [1] row_end, [2] nqg (0 = stop)
    uint64_t* full_bar = item + 4;
    uint64_t* empty_bar = full_bar + kStages;
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(empty_bar + kStages);

    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t nbox = dq / 32;
    const unsigned long long total_items = a.counters[1];
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], kConsumers);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();

    constexpr uint32_t nthreads_c = kConsumers * 32;
    const Consumer con(warp < kConsumers ? warp : 0, lane, stage_base, q_s, dq, xchg);
    auto row_key = [&](uint64_t r) { return a.row_map[r]; };

    uint32_t it = 0;  // ring position (producer and consumers walk the same sequence)
    for (;;) {
        if (tid == 0) {
            const unsigned long long w = *abort_flag ? total_items : atomicAdd(&a.counters[0], 1ull);
            if (w >= total_items) {
                item[2] = 0;
            } else {
                const uint32_t wi = static_cast<uint32_t>(w);
                uint32_t lo = 0, hi = a.nlist;  // last l with item_off[l] <= wi
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (a.item_off[mid] <= wi) lo = mid; else hi = mid;
                }
                const uint32_t l = lo;
                const uint32_t local = wi - a.item_off[l];
                const uint32_t nql = a.list_cnt[l];
                const uint32_t groups = (nql + QB - 1) / QB;
                const uint32_t chunk = local / groups, grp = local % groups;
                const uint64_t rb = a.offsets[l] + static_cast<uint64_t>(chunk) * kChunkRows;
                const uint64_t le = a.offsets[l + 1];
                item[0] = rb;
                item[1] = (rb + kChunkRows) < le ? (rb + kChunkRows) : le;
                const uint32_t q0 = grp * QB;
                const uint32_t nqg = (nql - q0) < static_cast<uint32_t>(QB) ? (nql - q0) : static_cast<uint32_t>(QB);
                item[2] = nqg;
                for (uint32_t b = 0; b < static_cast<uint32_t>(QB); ++b) {
                    const uint32_t src = a.list_qoff[l] + q0 + b;
                    qid[b] = b < nqg ? a.list_q[src] : 0u;
                    slot[b] = b < nqg ? a.list_slot[src] + chunk : 0u;
                }
            }
        }
        __syncthreads();
        const uint32_t nqg = static_cast<uint32_t>(item[2]);
        if (nqg == 0) break;
        const uint64_t row_begin = item[0], row_end = item[1];
        const uint32_t ntiles = static_cast<uint32_t>((row_end - row_begin + kTileRows - 1) / kTileRows);

        if (warp == kConsumers) {
            // ---------------- producer ----------------
            if (lane == 0) {
                const uint64_t policy = l2_policy_evict_first();
                bool stop = false;
                for (uint32_t t = 0; t < ntiles && !stop; ++t) {
                    const int32_t y = static_cast<int32_t>(row_begin + static_cast<uint64_t>(t) * kTileRows);
                    for (uint32_t bx = 0; bx < nbox; ++bx) {
                        const uint32_t s = it & (kStages - 1), u = it / kStages;
                        if (*abort_flag) {
                            stop = true;
                            break;
                        }
                        if (u > 0 && !mbar_wait_bounded(&empty_bar[s], (u - 1) & 1u, kWaitBudgetCycles)) {
                            *abort_flag = 1;
                            record_status(a.status, kStatusTimeout);
                            stop = true;
                            break;
                        }
                        mbar_arrive_expect_tx(&full_bar[s], kStageBytes);
                        tma_load_2d_hint(stage_base + static_cast<size_t>(s) * kStageBytes, &tmap, &full_bar[s],
                                         static_cast<int32_t>(bx * 32), y, policy);
                        ++it;
                    }
                }
            }
            it = __shfl_sync(0xffffffffu, it, 0);
        } else {
            // ---------------- consumers ----------------
            for (uint32_t i = tid; i < static_cast<uint32_t>(QB) * dq; i += nthreads_c) {
                const uint32_t b = i / dq, d = i - b * dq;
                q_s[i] = b < nqg ? a.queries[static_cast<uint64_t>(qid[b]) * dq + d] : 0.0f;
            }
            if (tid < static_cast<uint32_t>(QB)) {
                cnt[tid] = 0;
                thr[tid] = 0ull;
            }
            named_bar_sync(1, nthreads_c);
            float acc[4][Consumer::QW];
            for (uint32_t t = 0; t < ntiles; ++t) {
                con.accumulate(acc, nbox, it, full_bar, empty_bar, abort_flag, a.status);
                con.insert(acc, row_begin + static_cast<uint64_t>(t) * kTileRows, row_end, nqg, row_key, thr, cnt, cand,
                           cap, a.status);
                scan_flush<QB, kNcw>(t + 1 == ntiles, nqg, k, cap, warp, lane, cnt, thr, cand, hist);
            }
            for (uint32_t b = warp; b < nqg; b += kConsumers) {
                const uint32_t n = cnt[b] < k ? cnt[b] : k;
                uint64_t* dst = a.ws + static_cast<uint64_t>(slot[b]) * k;
                const uint64_t* src = cand + static_cast<size_t>(b) * cap;
                for (uint32_t j = lane; j < k; j += 32) dst[j] = j < n ? src[j] : 0ull;
            }
        }
        __syncthreads();  // the item's shared state is consumed before the next fetch
    }
    if (warp == kConsumers && lane == 0) {
        const uint32_t used = it < static_cast<uint32_t>(kStages) ? it : kStages;
        for (uint32_t s = 0; s < used; ++s) {
            const uint32_t uses = (it - s + kStages - 1) / kStages;
            if (!mbar_wait_bounded(&full_bar[s], (uses - 1) & 1u, kWaitBudgetCycles)) record_status(a.status, kStatusTimeout);
        }
    }
}

// ------------------------------------------------------------------------------------------
// 4. Merge: per query, the k best keys of its slots, sorted; unused result slots (0, 0.0f).
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(512)
    ivf_merge_kernel(const uint64_t* __restrict__ ws, const uint32_t* __restrict__ q_slot_off, uint32_t k,
                     uint64_t* __restrict__ idx_out, float* __restrict__ sim_out, uint32_t* __restrict__ count_out) {
    __shared__ BlockSelectScratch s;
    extern __shared__ uint64_t sorted[];
    const uint32_t q = blockIdx.x;
    const uint64_t* keys = ws + static_cast<uint64_t>(q_slot_off[q]) * k;
    const uint64_t n = static_cast<uint64_t>(q_slot_off[q + 1] - q_slot_off[q]) * k;
    if (threadIdx.x == 0) s.count = 0;
    __syncthreads();
    uint32_t local = 0;
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) local += keys[i] != 0ull;
    atomicAdd(&s.count, local);
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
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t key = keys[i];
            if (key != 0ull && key >= kth) {
                const uint32_t pos = atomicAdd(&s.count, 1u);
                if (pos < kk) sorted[pos] = key;
            }
        }
        __syncthreads();
        for (uint32_t i = kk + threadIdx.x; i < p2; i += blockDim.x) sorted[i] = 0ull;
        __syncthreads();
        block_bitonic_sort_desc(sorted, p2);
    }
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
        idx_out[static_cast<uint64_t>(q) * k + j] = j < kk ? key_row(sorted[j]) : 0;
        sim_out[static_cast<uint64_t>(q) * k + j] = j < kk ? key_score(sorted[j]) : 0.0f;
    }
    if (threadIdx.x == 0 && count_out) count_out[q] = kk;
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
namespace {

template <class T>
int grow(T*& p, size_t& cap, size_t n, const char* what) {
    if (n <= cap && p) return NNDEX_OK;
    cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return cuda_error(e, what);
    cap = n;
    return NNDEX_OK;
}

size_t ivf_scan_smem(uint32_t qb, uint32_t dq, uint32_t cap) {
    const size_t consumers = scan_consumers(qb, kNcw);
    size_t b = 1024;
    b += static_cast<size_t>(kStages) * kStageBytes;
    b += static_cast<size_t>(qb) * dq * 4;
    b += static_cast<size_t>(qb) * cap * 8;
    b += consumers * 32 * scan_xchg_per_lane(qb) * 4;
    b += consumers * 256 * 4;
    b += qb * 8 + (3 * qb + (qb & 1)) * 4;
    b += 4 * 8 + kStages * 16 + 16;
    return b;
}

template <int QB>
cudaError_t launch_scan(const CUtensorMap& tmap, const IvfScanArgs& a, uint32_t grid, size_t smem, cudaStream_t s) {
    auto kern = ivf_scan_kernel<QB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    kern<<<grid, ScanShape<QB, kNcw>::kThreads, smem, s>>>(tmap, a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace

int ivf_search(CudaIndex& ix, uint32_t nq, uint32_t k, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt,
               cudaStream_t s) {
    const IvfIndex& v = *ix.ivf;
    IvfScratch& w = ix.ivf_scratch;
    const uint32_t nlist = static_cast<uint32_t>(v.nlist);
    uint64_t np64 = w.nprobe ? w.nprobe : ivf_choose_nprobe(v.nlist, k, ix.rows);
    np64 = std::max<uint64_t>(1, std::min<uint64_t>(np64, v.nlist));
    const uint32_t np = static_cast<uint32_t>(np64);
    const uint32_t dq = static_cast<uint32_t>(ix.ds);
    // Queries per work item from the average number of queries probing a list.
    const double avg_q = static_cast<double>(nq) * np / nlist;
    uint32_t qb = avg_q >= 12.0 ? 16 : (avg_q >= 6.0 ? 8 : 4);
    const uint32_t cap = ((k + 2 * kTileRows) + 31) / 32 * 32;
    while (qb > 4 && ivf_scan_smem(qb, dq, cap) > ix.smem_optin) qb >>= 1;
    const size_t smem = ivf_scan_smem(qb, dq, cap);
    if (smem > ix.smem_optin)
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: IVF scan needs %zu bytes of shared memory", smem);
    if (static_cast<size_t>(ix.ds) * 4 + static_cast<size_t>(nlist) * 8 > ix.smem_optin)
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: IVF probe shared memory above the limit");
    const uint64_t max_chunks = (v.max_list + kChunkRows - 1) / kChunkRows;
    int st;
    // Sub-batches so the slot workspace (Σ slots × k keys) stays bounded.
    const uint64_t ws_budget = 256ull << 20;
    uint64_t per_query = std::max<uint64_t>(1, static_cast<uint64_t>(np) * max_chunks * k * 8);
    uint32_t sub = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(nq, ws_budget / per_query)));
    if ((st = grow(w.d_probes, w.cap_probes, static_cast<size_t>(sub) * np, "IVF probe buffer"))) return st;
    if ((st = grow(w.d_list_cnt, w.cap_list_cnt, nlist, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_fill, w.cap_list_fill, nlist, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_qoff, w.cap_list_qoff, nlist + 1, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_item_off, w.cap_item_off, nlist + 1, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_q, w.cap_list_q, static_cast<size_t>(sub) * np, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_slot, w.cap_list_slot, static_cast<size_t>(sub) * np, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_q_slot_off, w.cap_q_slot_off, sub + 1, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_counters, w.cap_counters, 6, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_ws, w.cap_ws, static_cast<size_t>(sub) * np * max_chunks * k, "IVF slot workspace"))) return st;
    IvfScanArgs a;
    a.dq = dq;
    a.k = k;
    a.cap = cap;
    a.nlist = nlist;
    a.offsets = v.d_offsets;
    a.row_map = v.d_row_map;
    a.list_cnt = w.d_list_cnt;
    a.list_qoff = w.d_list_qoff;
    a.item_off = w.d_item_off;
    a.list_q = w.d_list_q;
    a.list_slot = w.d_list_slot;
    a.counters = w.d_counters;
    a.ws = w.d_ws;
    a.status = ix.d_status;
    const size_t probe_smem = static_cast<size_t>(ix.ds) * 4 + static_cast<size_t>(nlist) * 8;
    cudaFuncSetAttribute(ivf_probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(probe_smem));
    uint32_t p2 = 1;
    while (p2 < k) p2 <<= 1;
    cudaMemsetAsync(w.d_counters, 0, 6 * sizeof(unsigned long long), s);
    for (uint32_t q0 = 0; q0 < nq; q0 += sub) {
        const uint32_t n = std::min(sub, nq - q0);
        const float* qn = ix.d_qn + static_cast<uint64_t>(q0) * ix.ds;
        cudaMemsetAsync(w.d_list_cnt, 0, nlist * sizeof(uint32_t), s);
        cudaMemsetAsync(w.d_list_fill, 0, nlist * sizeof(uint32_t), s);
        ivf_probe_kernel<<<n, 256, probe_smem, s>>>(qn, dq, static_cast<uint32_t>(ix.dp), v.d_cent_t, v.nlist_pad, nlist,
                                                    np, w.d_probes);
        ivf_plan_kernel<<<1, 1024, 0, s>>>(w.d_probes, n, np, nlist, v.d_offsets, qb, w.d_list_cnt, w.d_list_fill,
                                           w.d_list_qoff, w.d_item_off, w.d_list_q, w.d_list_slot, w.d_q_slot_off,
                                           w.d_counters);
        count_launch(2);
        a.queries = qn;
        cudaError_t e;
        cudaEvent_t ev_a = nullptr;
        ix.scan_event_begin(s, ev_a);
        switch (qb) {
            case 16: e = launch_scan<16>(v.tmap_reordered, a, static_cast<uint32_t>(ix.sm_count), smem, s); break;
            case 8: e = launch_scan<8>(v.tmap_reordered, a, static_cast<uint32_t>(ix.sm_count), smem, s); break;
            default: e = launch_scan<4>(v.tmap_reordered, a, static_cast<uint32_t>(ix.sm_count), smem, s); break;
        }
        ix.scan_event_end(s, ev_a);
        if (e != cudaSuccess) return cuda_error(e, "IVF scan launch");
        ivf_merge_kernel<<<n, 512, p2 * sizeof(uint64_t), s>>>(w.d_ws, w.d_q_slot_off, k, o_idx + static_cast<uint64_t>(q0) * k,
                                                               o_sim + static_cast<uint64_t>(q0) * k,
                                                               o_cnt ? o_cnt + q0 : nullptr);
        count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "IVF merge launch");
        ix.stats.kernel_launches += 4;
    }
    if (!w.h_probed && cudaMallocHost(&w.h_probed, 3 * sizeof(unsigned long long)) != cudaSuccess)
        return set_error(NNDEX_ERR_OUT_OF_MEMORY, "cuda execution error: pinned allocation failed");
    cudaMemcpyAsync(w.h_probed, w.d_counters + 3, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    ix.stats.path = 4;
    ix.stats.nprobe = np;
    return NNDEX_OK;
}

}  // namespace nndex
