// ivf_search.cu — K8/K9: IVF probe and the ragged list scan with exact FP32 rerank.
//
// Replaces candidate_clusters(_batch) (src/approx.rs:159-300) and search_approx /
// search_batch_approx (src/cpu.rs:425-502). A batch runs as six launches and no host round trip:
//   1. probe (two launches): per query, dot_small against every centroid (FP64 in index order, f32
//      result — the reference's value; up to 8 queries share each read of a centroid) and the nprobe
//      best clusters (score desc, lower index on ties).
//   2. plan (a one-block scan, then one warp per query): the (list, query) pairs grouped by list,
//      each list cut into chunks of at most kChunkRows rows, and work items (list chunk × group of up
//      to QB queries probing it), with every (query, list chunk) owning one output slot of k keys.
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
constexpr int kStages = 4;              // ring depth of the list scan

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
// 1. Probe, in two launches.
//    (a) Scores: a block scores 256 centroids against up to 8 queries (FP64 FMA in index order, f32
//        result, the queries held as doubles in shared memory), so each centroid read from L2
//        serves 8 queries and the grid (query groups × centroid chunks) fills every SM.
//    (b) Selection: one warp per query reads its scores (from L2) and selects its nprobe best lists
//        (a radix select over the keys (score, list)), writes them, and counts them into the plan:
//        queries per list, the query's output slots (one per chunk of a probed list), probed rows.
// ------------------------------------------------------------------------------------------
// The k-th largest of the n distinct keys (score, index i) of scores[0, n), by one warp (8 passes of
// 8 bits; `hist` 256 words of the warp's own).
NNDEX_DEVICE_INLINE uint64_t warp_radix_kth(const float* scores, uint32_t n, uint32_t k, uint32_t* hist,
                                            uint32_t lane) {
    uint64_t prefix = 0, mask = 0;
    uint32_t krem = k;
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (uint32_t i = lane; i < 256; i += 32) hist[i] = 0;
        __syncwarp();
        for (uint32_t i = lane; i < n; i += 32) {
            const uint64_t key = make_key(scores[i], i);
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncwarp();
        // lane L owns bins 255 − 8L down to 248 − 8L: counts above a bin accumulate from lane 0
        uint32_t c[8], local = 0;
#pragma unroll
        for (uint32_t b = 0; b < 8; ++b) {
            c[b] = hist[255u - (lane * 8u + b)];
            local += c[b];
        }
        uint32_t incl = local;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += x;
        }
        const uint32_t excl = incl - local;
        const uint32_t owner = __ffs(__ballot_sync(0xFFFFFFFFu, excl < krem && krem <= incl)) - 1;
        uint32_t bin = 0, above = excl, in_bin = 0;
        if (lane == owner) {
#pragma unroll
            for (uint32_t b = 0; b < 8; ++b) {
                if (above + c[b] >= krem) {
                    bin = 255u - (lane * 8u + b);
                    in_bin = c[b];
                    break;
                }
                above += c[b];
            }
        }
        bin = __shfl_sync(0xFFFFFFFFu, bin, owner);
        above = __shfl_sync(0xFFFFFFFFu, above, owner);
        in_bin = __shfl_sync(0xFFFFFFFFu, in_bin, owner);
        prefix |= static_cast<uint64_t>(bin) << shift;
        mask |= 0xFFull << shift;
        krem -= above;
        __syncwarp();
        if (in_bin == krem) {
            // every key of this bin is selected: the k-th is the smallest of them
            uint64_t m = ~0ull;
            for (uint32_t i = lane; i < n; i += 32) {
                const uint64_t key = make_key(scores[i], i);
                if ((key & mask) == prefix && key < m) m = key;
            }
            return warp_min_u64(m);
        }
    }
    return prefix;
}

constexpr uint32_t kProbeCentroids = 256;  // centroids per scoring block
constexpr uint32_t kProbeThreads = 128;    // two centroids per thread

static size_t probe_smem(uint32_t qb, uint64_t dp) { return static_cast<size_t>(qb) * dp * 8; }

// Each thread scores two centroids (c and c + 128) against the block's QB queries: every query
// value read from shared memory feeds two FMAs (one FMA per read left the kernel waiting on its
// shared-memory loads, the FP64 pipe 36 % busy).
template <int QB>
__global__ void __launch_bounds__(kProbeThreads)
    ivf_probe_score_kernel(const float* __restrict__ queries, uint32_t nq, uint32_t ds, uint32_t dp,
                           const float* __restrict__ cent_t, uint64_t ct_stride, uint32_t nlist,
                           float* __restrict__ scores) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    double* qd = reinterpret_cast<double*>(smem_raw);  // [dp][QB]
    const uint32_t q0 = blockIdx.x * QB;
    const uint32_t nb = (nq - q0) < QB ? (nq - q0) : QB;
    for (uint32_t i = threadIdx.x; i < dp * QB; i += blockDim.x) {
        const uint32_t d = i / QB, j = i % QB;
        qd[i] = j < nb ? static_cast<double>(queries[static_cast<uint64_t>(q0 + j) * ds + d]) : 0.0;
    }
    __syncthreads();
    const uint32_t c0 = blockIdx.y * kProbeCentroids + threadIdx.x, c1 = c0 + kProbeThreads;
    if (c0 >= nlist) return;
    const bool two = c1 < nlist;
    double a0[QB], a1[QB];
#pragma unroll
    for (int j = 0; j < QB; ++j) a0[j] = a1[j] = 0.0;
    const float* col0 = cent_t + c0;
    const float* col1 = cent_t + (two ? c1 : c0);
#pragma unroll 4
    for (uint32_t d = 0; d < dp; ++d) {
        const double v0 = static_cast<double>(__ldg(col0 + static_cast<uint64_t>(d) * ct_stride));
        const double v1 = static_cast<double>(__ldg(col1 + static_cast<uint64_t>(d) * ct_stride));
        const double* qv = qd + static_cast<size_t>(d) * QB;
#pragma unroll
        for (int j = 0; j < QB; ++j) {
            const double x = qv[j];
            a0[j] = fma(v0, x, a0[j]);
            a1[j] = fma(v1, x, a1[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < QB; ++j)
        if (j < static_cast<int>(nb)) {
            float* row = scores + static_cast<uint64_t>(q0 + j) * nlist;
            row[c0] = fold_zero(__double2float_rn(a0[j]));
            if (two) row[c1] = fold_zero(__double2float_rn(a1[j]));
        }
}

__global__ void __launch_bounds__(256)
    ivf_probe_select_kernel(const float* __restrict__ scores, uint32_t nq, uint32_t nlist, uint32_t np,
                            const uint32_t* __restrict__ offsets, uint32_t* __restrict__ probes,
                            uint32_t* __restrict__ list_cnt, uint32_t* __restrict__ q_slot_off,
                            unsigned long long* __restrict__ counters) {
    __shared__ uint32_t hist_all[8][256];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t q = blockIdx.x * 8 + warp;
    if (q >= nq) return;
    const float* sq = scores + static_cast<uint64_t>(q) * nlist;
    const uint64_t kth = np < nlist ? warp_radix_kth(sq, nlist, np, hist_all[warp], lane) : 0ull;
    uint32_t base = 0, slots = 0;
    unsigned long long rows = 0;
    for (uint32_t c0 = 0; c0 < nlist; c0 += 32) {
        const uint32_t c = c0 + lane;
        const bool take = c < nlist && make_key(sq[c], c) >= kth;
        const uint32_t ballot = __ballot_sync(0xFFFFFFFFu, take);
        if (take) {
            const uint32_t pos = base + __popc(ballot & ((1u << lane) - 1u));
            if (pos < np) {
                probes[static_cast<uint64_t>(q) * np + pos] = c;
                atomicAdd(&list_cnt[c], 1u);
                const uint32_t len = offsets[c + 1] - offsets[c];
                slots += (len + kChunkRows - 1) / kChunkRows;
                rows += len;
            }
        }
        base += __popc(ballot);
    }
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1) {
        slots += __shfl_xor_sync(0xFFFFFFFFu, slots, o);
        rows += __shfl_xor_sync(0xFFFFFFFFu, rows, o);
    }
    if (lane == 0) {
        q_slot_off[q] = slots;
        atomicAdd(&counters[3], rows);  // zeroed once per search: Σ over sub-batches
    }
}

// ------------------------------------------------------------------------------------------
// 2. Plan, from the probe's counts. (a) One block: per list its work items (chunks × groups of qb
//    queries) and gathered query blocks, and the exclusive scans that place each list's queries,
//    items and blocks and each query's slots. (b) One warp per query: its (list, query) pairs
//    written into their lists, each with the query's slot of the list's first chunk.
//    counters[0] work-item counter (the scan's), [1] items, [2] slots; summed over the sub-batches of
//    a search: [3] Σ rows probed per query, [4] rows streamed by the scan, [5] rows of probed lists;
//    [6] gathered query blocks (qblock_off given: the tensor-core scan's groups of qb queries).
//    Groups of a list are consecutive blocks from qblock_off[l].
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024)
    ivf_plan_scan_kernel(uint32_t nq, uint32_t nlist, const uint32_t* __restrict__ offsets, uint32_t qb,
                         const uint32_t* __restrict__ list_cnt, uint32_t* __restrict__ list_qoff,
                         uint32_t* __restrict__ item_off, uint32_t* __restrict__ q_slot_off,
                         unsigned long long* __restrict__ counters, uint32_t* __restrict__ qblock_off) {
    __shared__ uint32_t part[1024];
    unsigned long long my_stream = 0, my_union = 0;
    for (uint32_t l = threadIdx.x; l < nlist; l += blockDim.x) {
        const uint32_t c = list_cnt[l];
        const uint32_t groups = (c + qb - 1) / qb;
        const uint32_t len = offsets[l + 1] - offsets[l];
        item_off[l] = (len + kChunkRows - 1) / kChunkRows * groups;
        list_qoff[l] = c;
        if (qblock_off) qblock_off[l] = groups;
        my_stream += static_cast<unsigned long long>(len) * groups;
        my_union += c ? len : 0u;
    }
    atomicAdd(&counters[4], my_stream);
    atomicAdd(&counters[5], my_union);
    __syncthreads();
    block_exclusive_scan(list_qoff, nlist, part);
    block_exclusive_scan(item_off, nlist, part);
    block_exclusive_scan(q_slot_off, nq, part);
    if (qblock_off) block_exclusive_scan(qblock_off, nlist, part);
    if (threadIdx.x == 0) {
        counters[0] = 0;
        counters[1] = item_off[nlist];
        counters[2] = q_slot_off[nq];
        if (qblock_off) counters[6] = qblock_off[nlist];
    }
}

__global__ void __launch_bounds__(256)
    ivf_plan_fill_kernel(const uint32_t* __restrict__ probes, uint32_t nq, uint32_t np,
                         const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ list_qoff,
                         uint32_t* __restrict__ list_fill, const uint32_t* __restrict__ q_slot_off,
                         uint32_t* __restrict__ list_q, uint32_t* __restrict__ list_slot) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (q >= nq) return;
    uint32_t run = q_slot_off[q];  // the query's slots, its probed lists' chunks in probe order
    for (uint32_t j0 = 0; j0 < np; j0 += 32) {
        const uint32_t j = j0 + lane;
        const bool on = j < np;
        const uint32_t l = on ? probes[static_cast<uint64_t>(q) * np + j] : 0u;
        const uint32_t c = on ? (offsets[l + 1] - offsets[l] + kChunkRows - 1) / kChunkRows : 0u;
        uint32_t incl = c;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += x;
        }
        if (on) {
            const uint32_t pos = list_qoff[l] + atomicAdd(&list_fill[l], 1u);
            list_q[pos] = q;
            list_slot[pos] = run + incl - c;
        }
        run += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
}

// ------------------------------------------------------------------------------------------
// 3. Ragged list scan (persistent). Producer warp: TMA of 128-row × 128-byte boxes of the
//    reordered rows. Consumer warps: the FP32 scan's wide consumer, FMA order and addition tree.
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

// Consumer warps of the list scan per queries per item: ScanConsumerWide (16 rows × all the item's
// queries per warp, the FP32 scan's FMA order and addition tree); 8 warps of 128-row tiles at 16
// queries, 16 warps of 256-row tiles (two 128-row boxes per slab) at 4 or 8.
template <int QB>
struct IvfScanShape {
    static constexpr int kW = QB >= 16 ? 8 : 16;
    static constexpr int kThreads = (kW + 1) * 32;
};

template <int QB>
__global__ void __launch_bounds__(IvfScanShape<QB>::kThreads, 1)
    ivf_scan_kernel(const __grid_constant__ CUtensorMap tmap, const IvfScanArgs a) {
    constexpr int W = IvfScanShape<QB>::kW;
    using Consumer = ScanConsumerWide<QB, W, kStages>;
    constexpr int TR = Consumer::kTileRows;
    constexpr uint32_t kStage = Consumer::kStageBytes;
    constexpr uint32_t kBoxes = TR / 128;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* stage_base = align_1024(smem_raw);
    const uint32_t dq = a.dq, cap = a.cap, k = a.k;
    float* q_s = reinterpret_cast<float*>(stage_base + static_cast<size_t>(kStages) * kStage);
    uint64_t* cand = reinterpret_cast<uint64_t*>(q_s + static_cast<size_t>(QB) * dq);
    uint32_t* hist = reinterpret_cast<uint32_t*>(cand + static_cast<size_t>(QB) * cap);
    uint64_t* thr = reinterpret_cast<uint64_t*>(hist + W * 256);
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
            mbar_init(&empty_bar[s], W * 32);  // every consumer lane releases
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();

    constexpr uint32_t nthreads_c = W * 32;
    const Consumer con(warp < static_cast<uint32_t>(W) ? warp : 0, lane, stage_base, q_s);
    auto row_key = [&](uint64_t r) { return a.row_map[r]; };

    // Producer and consumers walk the same sequence of ring positions across items.
    uint32_t it = 0;
    RingPos<kStages> pos;
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
        const uint32_t ntiles = static_cast<uint32_t>((row_end - row_begin + TR - 1) / TR);

        if (warp == static_cast<uint32_t>(W)) {
            // ---------------- producer ----------------
            if (lane == 0) {
                const uint64_t policy = l2_policy_evict_first();
                bool stop = false;
                for (uint32_t t = 0; t < ntiles && !stop; ++t) {
                    const int32_t y = static_cast<int32_t>(row_begin + static_cast<uint64_t>(t) * TR);
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
                        mbar_arrive_expect_tx(&full_bar[s], kStage);
#pragma unroll
                        for (uint32_t h = 0; h < kBoxes; ++h)
                            tma_load_2d_hint(stage_base + static_cast<size_t>(s) * kStage + h * 128 * 128, &tmap,
                                             &full_bar[s], static_cast<int32_t>(bx * 32),
                                             y + static_cast<int32_t>(h * 128), policy);
                        ++it;
                    }
                }
            }
            it = __shfl_sync(0xffffffffu, it, 0);
        } else {
            // ---------------- consumers ----------------
            for (uint32_t i = tid; i < static_cast<uint32_t>(QB) * dq; i += nthreads_c) {
                const uint32_t b = i / dq, d = i - b * dq;
                q_s[Consumer::q_slab_index(b, d)] = b < nqg ? a.queries[static_cast<uint64_t>(qid[b]) * dq + d] : 0.0f;
            }
            if (tid < static_cast<uint32_t>(QB)) {
                cnt[tid] = 0;
                thr[tid] = 0ull;
            }
            named_bar_sync(1, nthreads_c);
            float acc[4][QB];
            for (uint32_t t = 0; t < ntiles; ++t) {
                con.accumulate(acc, nbox, pos, full_bar, empty_bar, abort_flag, a.status);
                con.insert(acc, row_begin + static_cast<uint64_t>(t) * TR, row_end, nqg, row_key, thr, cnt, cand, cap,
                           a.status);
                scan_flush_g<QB, W, TR>(t + 1 == ntiles, nqg, k, cap, warp, lane, cnt, thr, cand, hist);
            }
            for (uint32_t b = warp; b < nqg; b += W) {
                const uint32_t n = cnt[b] < k ? cnt[b] : k;
                uint64_t* dst = a.ws + static_cast<uint64_t>(slot[b]) * k;
                const uint64_t* src = cand + static_cast<size_t>(b) * cap;
                for (uint32_t j = lane; j < k; j += 32) dst[j] = j < n ? src[j] : 0ull;
            }
        }
        __syncthreads();  // the item's shared state is consumed before the next fetch
    }
    if (warp == static_cast<uint32_t>(W) && lane == 0) {
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
    local = __reduce_add_sync(0xffffffffu, local);
    if (lane_id() == 0) atomicAdd(&s.count, local);
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
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
        idx_out[static_cast<uint64_t>(q) * k + j] = j < out_n ? key_row(sorted[j]) : 0;
        sim_out[static_cast<uint64_t>(q) * k + j] = j < out_n ? key_score(sorted[j]) : 0.0f;
    }
    if (threadIdx.x == 0 && count_out) count_out[q] = out_n;
}

// ------------------------------------------------------------------------------------------
// Tensor-core list scan helpers.
// ------------------------------------------------------------------------------------------
// One block per list: its probing queries in groups of 128 (one gathered block each, consecutive from
// qblock_off[l]): their BF16 rows (zero past the group's end), query ids (0xFFFFFFFF: none) and the
// query's output slot for the list's chunk 0.
__global__ void __launch_bounds__(256)
    ivf_gather_tc_kernel(const __nv_bfloat16* __restrict__ q16, uint32_t kb, const uint32_t* __restrict__ list_cnt,
                         const uint32_t* __restrict__ list_qoff, const uint32_t* __restrict__ list_q,
                         const uint32_t* __restrict__ list_slot, const uint32_t* __restrict__ qblock_off,
                         __nv_bfloat16* __restrict__ g16, uint32_t* __restrict__ lane_qid,
                         uint32_t* __restrict__ lane_slot, const uint32_t* __restrict__ item_off,
                         uint32_t* __restrict__ item_list) {
    const uint32_t l = blockIdx.x;
    const uint32_t cnt = list_cnt[l];
    if (cnt == 0) return;
    // the list of each of this list's work items (so a scan CTA finds its list with one load)
    for (uint32_t i = item_off[l] + threadIdx.x; i < item_off[l + 1]; i += blockDim.x) item_list[i] = l;
    const uint32_t n = (cnt + 127) / 128 * 128;
    const uint64_t row0 = static_cast<uint64_t>(qblock_off[l]) * 128;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, nwarps = blockDim.x >> 5;
    const uint32_t chunks = kb / 8;  // 16-byte chunks of a row
    for (uint32_t j = warp; j < n; j += nwarps) {
        const uint64_t row = row0 + j;
        uint4* dst = reinterpret_cast<uint4*>(g16 + row * kb);
        if (j < cnt) {
            const uint32_t src = list_qoff[l] + j;
            const uint32_t q = list_q[src];
            const uint4* from = reinterpret_cast<const uint4*>(q16 + static_cast<uint64_t>(q) * kb);
            for (uint32_t c = lane; c < chunks; c += 32) dst[c] = from[c];
            if (lane == 0) {
                lane_qid[row] = q;
                lane_slot[row] = list_slot[src];
            }
        } else {
            for (uint32_t c = lane; c < chunks; c += 32) dst[c] = make_uint4(0u, 0u, 0u, 0u);
            if (lane == 0) {
                lane_qid[row] = 0xFFFFFFFFu;
                lane_slot[row] = 0;
            }
        }
    }
}

// Pass-2 thresholds by query: the exact k-th score of pass 1, or +inf for a certified query.
__global__ void ivf_pass2_thr_kernel(const uint32_t* __restrict__ cert, const float* __restrict__ kth, uint32_t n,
                                     float* __restrict__ thr) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) thr[q] = cert[q] ? INFINITY : kth[q];
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
namespace {

template <class T>
int grow(T*& p, size_t& cap, size_t n, const char* what) {
    if (n <= cap && p) return NNDEX_OK;
    bump_alloc_epoch();
    cap = 0;
    void* raw = p;
    cudaError_t e = take_injected_alloc_failure() ? cudaErrorMemoryAllocation
                                                  : regrow_raw(&raw, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaErrorMemoryAllocation && raw) cudaFree(raw);  // an injected failure frees it too
    if (e != cudaSuccess) {
        p = nullptr;
        return cuda_error(e, what);
    }
    p = static_cast<T*>(raw);
    cap = n;
    return NNDEX_OK;
}

// Tile rows of the list scan at qb queries per item (IvfScanShape).
uint32_t ivf_scan_tile_rows(uint32_t qb) { return qb >= 16 ? 8 * 16 : 16 * 16; }

size_t ivf_scan_smem(uint32_t qb, uint32_t dq, uint32_t cap) {
    const uint32_t w = qb >= 16 ? 8 : 16;
    size_t b = 1024;
    b += static_cast<size_t>(kStages) * ivf_scan_tile_rows(qb) * 128;
    b += static_cast<size_t>(qb) * dq * 4;
    b += static_cast<size_t>(qb) * cap * 8;
    b += static_cast<size_t>(w) * 256 * 4;
    b += qb * 8 + (3 * qb + (qb & 1)) * 4;
    b += 4 * 8 + kStages * 16 + 16;
    return b;
}

template <int QB>
cudaError_t launch_scan(const CUtensorMap& tmap, const IvfScanArgs& a, uint32_t grid, size_t smem, cudaStream_t s) {
    auto kern = ivf_scan_kernel<QB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    kern<<<grid, IvfScanShape<QB>::kThreads, smem, s>>>(tmap, a);
    count_launch();
    return cudaGetLastError();
}

// The sampled pass-1 stride of the tensor-core list scan's rules.
uint32_t ivf_sampled_stride() {
    static const uint32_t sampled = [] {
        const char* v = getenv("NNDEX_IVF_TC_STRIDE");  // measurement override of the sampled stride
        const uint32_t x = v ? static_cast<uint32_t>(strtoul(v, nullptr, 10)) : 0u;
        return x >= 2 && x <= 16 ? x : 4u;
    }();
    return sampled;
}

// Queries per probe scoring block: the most (8, 4, 2 or 1) held as doubles in shared memory; 0 if
// not even one fits.
uint32_t probe_qb(uint64_t dp, size_t smem_optin) {
    for (uint32_t qb = 8; qb >= 1; qb >>= 1)
        if (probe_smem(qb, dp) <= smem_optin) return qb;
    return 0;
}

struct ProbeLaunch {
    const float* queries;
    uint32_t nq, ds, dp, nlist, np;
    const float* cent_t;
    uint64_t ct_stride;
    const uint32_t* offsets;
    float* scores;  // nq × nlist
    uint32_t* probes;
    uint32_t* list_cnt;
    uint32_t* q_slot_off;
    unsigned long long* counters;
};

template <int QB>
cudaError_t launch_probe_qb(const ProbeLaunch& a, cudaStream_t s) {
    auto kern = ivf_probe_score_kernel<QB>;
    const size_t smem = probe_smem(QB, a.dp);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const dim3 grid((a.nq + QB - 1) / QB, (a.nlist + kProbeCentroids - 1) / kProbeCentroids);
    kern<<<grid, kProbeThreads, smem, s>>>(a.queries, a.nq, a.ds, a.dp, a.cent_t, a.ct_stride, a.nlist, a.scores);
    return cudaGetLastError();
}

// Probe + plan of n queries: four launches (centroid scores, the selection with its counts, the
// plan's scans, the pairs).
cudaError_t launch_probe_plan(uint32_t pqb, const ProbeLaunch& a, uint32_t qb, IvfScratch& w, uint32_t* qblock_off,
                              cudaStream_t s) {
    if ((a.nlist + kProbeCentroids - 1) / kProbeCentroids > 65535u) return cudaErrorInvalidValue;
    cudaError_t e;
    switch (pqb) {
        case 8: e = launch_probe_qb<8>(a, s); break;
        case 4: e = launch_probe_qb<4>(a, s); break;
        case 2: e = launch_probe_qb<2>(a, s); break;
        case 1: e = launch_probe_qb<1>(a, s); break;
        default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    ivf_probe_select_kernel<<<(a.nq + 7) / 8, 256, 0, s>>>(a.scores, a.nq, a.nlist, a.np, a.offsets, a.probes,
                                                           a.list_cnt, a.q_slot_off, a.counters);
    ivf_plan_scan_kernel<<<1, 1024, 0, s>>>(a.nq, a.nlist, a.offsets, qb, w.d_list_cnt, w.d_list_qoff, w.d_item_off,
                                            w.d_q_slot_off, w.d_counters, qblock_off);
    ivf_plan_fill_kernel<<<(a.nq + 7) / 8, 256, 0, s>>>(a.probes, a.nq, a.np, a.offsets, w.d_list_qoff, w.d_list_fill,
                                                         w.d_q_slot_off, w.d_list_q, w.d_list_slot);
    count_launch(4);
    return cudaGetLastError();
}

template <class T>
int grow_pinned(T*& p, size_t& cap, size_t n, const char* what) {
    // geometric from 4,096 elements: releasing a pinned buffer waits for the device (in a serving
    // slot, for the other slots' batches too)
    if (n <= cap && p) return NNDEX_OK;
    bump_alloc_epoch();
    cudaFreeHost(p);
    p = nullptr;
    const size_t want = std::max<size_t>({n, cap * 2, 4096});
    cap = 0;
    cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&p), want * sizeof(T));
    if (e != cudaSuccess) return cuda_error(e, what);
    cap = want;
    return NNDEX_OK;
}

}  // namespace

int ivf_search(CudaIndex& ix, const float* queries, uint32_t nq, uint32_t k, uint64_t* o_idx, float* o_sim,
               uint32_t* o_cnt, cudaStream_t s) {
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
    auto cap_for = [&](uint32_t b) { return ((k + 2 * ivf_scan_tile_rows(b)) + 31) / 32 * 32; };
    while (qb > 4 && ivf_scan_smem(qb, dq, cap_for(qb)) > ix.smem_optin) qb >>= 1;
    const uint32_t cap = cap_for(qb);
    const size_t smem = ivf_scan_smem(qb, dq, cap);
    if (smem > ix.smem_optin)
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: IVF scan needs %zu bytes of shared memory", smem);
    const uint32_t pqb = probe_qb(ix.dp, ix.smem_optin);
    if (!pqb) return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: IVF probe shared memory above the limit");
    const uint64_t max_chunks = (v.max_list + kChunkRows - 1) / kChunkRows;
    int st;
    // Sub-batches so the slot workspace (Σ slots × k keys) stays bounded.
    const uint64_t ws_budget = 256ull << 20;
    uint64_t per_query = std::max<uint64_t>(1, static_cast<uint64_t>(np) * max_chunks * k * 8);
    uint32_t sub = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(nq, ws_budget / per_query)));
    if ((st = grow(w.d_probes, w.cap_probes, static_cast<size_t>(sub) * np, "IVF probe buffer"))) return st;
    if ((st = grow(w.d_pscore, w.cap_pscore, static_cast<size_t>(sub) * nlist, "IVF probe buffer"))) return st;
    if ((st = grow(w.d_list_cnt, w.cap_list_cnt, nlist, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_fill, w.cap_list_fill, nlist, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_qoff, w.cap_list_qoff, nlist + 1, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_item_off, w.cap_item_off, nlist + 1, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_q, w.cap_list_q, static_cast<size_t>(sub) * np, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_slot, w.cap_list_slot, static_cast<size_t>(sub) * np, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_q_slot_off, w.cap_q_slot_off, sub + 1, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_counters, w.cap_counters, 8, "IVF plan buffer"))) return st;
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
    uint32_t p2 = 1;
    while (p2 < k) p2 <<= 1;
    cudaMemsetAsync(w.d_counters, 0, 8 * sizeof(unsigned long long), s);
    for (uint32_t q0 = 0; q0 < nq; q0 += sub) {
        const uint32_t n = std::min(sub, nq - q0);
        const float* qn = queries + static_cast<uint64_t>(q0) * ix.ds;
        cudaMemsetAsync(w.d_list_cnt, 0, nlist * sizeof(uint32_t), s);
        cudaMemsetAsync(w.d_list_fill, 0, nlist * sizeof(uint32_t), s);
        const ProbeLaunch pl{qn,          n,          dq,           static_cast<uint32_t>(ix.dp), nlist, np,
                             v.d_cent_t,  v.nlist_pad, v.d_offsets, w.d_pscore, w.d_probes, w.d_list_cnt,
                             w.d_q_slot_off, w.d_counters};
        cudaError_t e = launch_probe_plan(pqb, pl, qb, w, nullptr, s);
        if (e != cudaSuccess) return cuda_error(e, "IVF probe launch");
        a.queries = qn;
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
        ix.stats.kernel_launches += 6;
    }
    if (!w.h_probed) bump_alloc_epoch();
    if (!w.h_probed && cudaMallocHost(&w.h_probed, 8 * sizeof(unsigned long long)) != cudaSuccess)
        return set_error(NNDEX_ERR_OUT_OF_MEMORY, "cuda execution error: pinned allocation failed");
    cudaMemcpyAsync(w.h_probed, w.d_counters + 3, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    ix.stats.path = 4;
    ix.stats.nprobe = np;
    return NNDEX_OK;
}

// Tensor-core list scan (path 5). Pass 1: the plan groups the queries probing each list by 128;
// each work item (list chunk × query group) runs the tensor-core scan in item mode over the list's
// reordered BF16 rows and leaves the k′ best upper bounds per (query, chunk) in its slot; the merge
// keeps the k′ best per query over its slots and K4 re-scores them exactly in FP32: the exact k-th
// score T, and a certificate when T beats the k′-th bound (no other probed row can reach the top k).
// Pass 2, for the other queries: every probed row whose bound reaches T, re-scored exactly. The
// result equals the FP32 list scan's (the same probed rows, the same exact scores, bit for bit).
//
// Everything is enqueued without a host round trip: the grid is the largest item count the plan
// can produce (its CTAs past the plan's own count return at once), the uncertified queries are
// compacted on the device (pass 2 returns at once when there are none), and the queries whose
// collection overflowed are compacted for ivf_finish_tc, which runs once the stream has completed.
int ivf_search_tc(CudaIndex& ix, uint32_t nq, uint32_t k, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt,
                  cudaStream_t s) {
    const IvfIndex& v = *ix.ivf;
    IvfScratch& w = ix.ivf_scratch;
    const uint32_t nlist = static_cast<uint32_t>(v.nlist);
    uint64_t np64 = w.nprobe ? w.nprobe : ivf_choose_nprobe(v.nlist, k, ix.rows);
    np64 = std::max<uint64_t>(1, std::min<uint64_t>(np64, v.nlist));
    const uint32_t np = static_cast<uint32_t>(np64);
    const CudaIndex::TcPlan plan = ix.plan_tc(k, false), plan2 = ix.plan_tc(0, false);
    if (plan.kp < k || !plan.stages || !plan2.stages) return ivf_search(ix, ix.d_qn, nq, k, o_idx, o_sim, o_cnt, s);
    const uint32_t kp = plan.kp;
    const uint32_t pqb = probe_qb(ix.dp, ix.smem_optin);
    if (!pqb) return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: IVF probe shared memory above the limit");
    const uint64_t max_chunks = (v.max_list + kChunkRows - 1) / kChunkRows;
    const uint64_t pairs = static_cast<uint64_t>(nq) * np;
    const uint64_t max_blocks = nlist + (pairs + 127) / 128;
    // Σ over lists of (query groups × chunks) ≤ (pairs / 128) · max_chunks + Σ chunks ≤ … + rows / chunk + nlist
    const uint64_t max_items = (pairs + 127) / 128 * max_chunks + ix.rows / kChunkRows + nlist + 1;
    if (max_items > 0x7FFFFFFFull)
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: IVF batch of %u queries × %u lists too large", nq, np);
    const uint32_t cap2 = kSecondPassCap;
    int st;
    if ((st = grow(w.d_probes, w.cap_probes, pairs, "IVF probe buffer"))) return st;
    if ((st = grow(w.d_pscore, w.cap_pscore, static_cast<size_t>(nq) * nlist, "IVF probe buffer"))) return st;
    if ((st = grow(w.d_list_cnt, w.cap_list_cnt, nlist, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_fill, w.cap_list_fill, nlist, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_qoff, w.cap_list_qoff, nlist + 1, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_item_off, w.cap_item_off, nlist + 1, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_qblock_off, w.cap_qblock_off, nlist + 1, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_q, w.cap_list_q, pairs, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_list_slot, w.cap_list_slot, pairs, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_q_slot_off, w.cap_q_slot_off, nq + 1, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_counters, w.cap_counters, 10, "IVF plan buffer"))) return st;
    if ((st = grow(w.d_ws, w.cap_ws, pairs * max_chunks * kp, "IVF slot workspace"))) return st;
    if ((st = grow(w.d_g16, w.cap_g16, max_blocks * 128 * v.kb16, "IVF query blocks"))) return st;
    if ((st = grow(w.d_lane_qid, w.cap_lane_qid, max_blocks * 128, "IVF query blocks"))) return st;
    if ((st = grow(w.d_lane_slot, w.cap_lane_slot, max_blocks * 128, "IVF query blocks"))) return st;
    if ((st = grow(w.d_item_list, w.cap_item_list, max_items, "IVF plan buffer"))) return st;
    if ((st = grow(ix.d_thr, ix.cap_thr, nq, "tc workspace"))) return st;
    if ((st = grow(ix.d_cand_idx, ix.cap_cand_idx, static_cast<size_t>(nq) * kp, "tc workspace"))) return st;
    if ((st = grow(ix.d_cand_sim, ix.cap_cand_sim, static_cast<size_t>(nq) * kp, "tc workspace"))) return st;
    if ((st = grow(ix.d_cand_cnt, ix.cap_cand_cnt, nq, "tc workspace"))) return st;
    if ((st = grow(ix.d_cert, ix.cap_cert, nq, "tc workspace"))) return st;
    if ((st = grow(ix.d_kth, ix.cap_kth, nq, "tc workspace"))) return st;
    if ((st = grow(ix.d_ids, ix.cap_ids, nq, "pass-2 buffer"))) return st;
    if ((st = grow(ix.d_q2_thr, ix.cap_q2_thr, nq, "pass-2 buffer"))) return st;
    if ((st = grow(ix.d_rows2, ix.cap_rows2, static_cast<size_t>(nq) * cap2, "pass-2 buffer"))) return st;
    if ((st = grow(ix.d_cnt2, ix.cap_cnt2, nq, "pass-2 buffer"))) return st;
    if ((st = grow(ix.d_ok2, ix.cap_ok2, nq, "pass-2 buffer"))) return st;
    if ((st = grow(ix.d_tcfail, ix.cap_tcfail, nq, "pass-2 buffer"))) return st;
    if ((st = grow(ix.d_rslots, ix.cap_rslots, static_cast<size_t>(nq) * rerank_chunks(cap2) * k, "pass-2 buffer")))
        return st;
    if ((st = ix.ensure_fbn())) return st;
    if (!w.h_probed) bump_alloc_epoch();
    if (!w.h_probed && cudaMallocHost(&w.h_probed, 8 * sizeof(unsigned long long)) != cudaSuccess)
        return set_error(NNDEX_ERR_OUT_OF_MEMORY, "cuda execution error: pinned allocation failed");

    // ---- probe + plan (groups of 128 queries) + gathered query blocks ----
    // [8] and [9]: the work-item counters of the two tensor-core passes
    cudaMemsetAsync(w.d_counters, 0, 10 * sizeof(unsigned long long), s);
    cudaMemsetAsync(w.d_list_cnt, 0, nlist * sizeof(uint32_t), s);
    cudaMemsetAsync(w.d_list_fill, 0, nlist * sizeof(uint32_t), s);
    const ProbeLaunch pl{ix.d_qn,   nq,          static_cast<uint32_t>(ix.ds), static_cast<uint32_t>(ix.dp),
                         nlist,      np,          v.d_cent_t,  v.nlist_pad, v.d_offsets, w.d_pscore, w.d_probes,
                         w.d_list_cnt, w.d_q_slot_off, w.d_counters};
    cudaError_t e = launch_probe_plan(pqb, pl, 128, w, w.d_qblock_off, s);
    if (e != cudaSuccess) return cuda_error(e, "IVF probe launch");
    ivf_gather_tc_kernel<<<nlist, 256, 0, s>>>(ix.d_q_bf16, static_cast<uint32_t>(v.kb16), w.d_list_cnt, w.d_list_qoff,
                                               w.d_list_q, w.d_list_slot, w.d_qblock_off, w.d_g16, w.d_lane_qid,
                                               w.d_lane_slot, w.d_item_off, w.d_item_list);
    count_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "IVF plan launch");

    // ---- pass 1 ----
    CUtensorMap tmap_q;
    if ((st = ix.encode_query_tmap(false, w.d_g16, static_cast<uint32_t>(max_blocks * 128), &tmap_q))) return st;
    cudaMemsetAsync(ix.d_thr, 0, nq * sizeof(unsigned long long), s);
    TcArgs a;
    a.tmap_q = &tmap_q;
    a.tmap_b = &v.tmap_reordered16;
    a.nranges = 1;
    a.stages = plan.stages;
    a.stream_a = plan.stream_a;
    a.items = static_cast<uint32_t>(max_items);
    ix.fill_tc_params(false, nq, 0, a.p);
    a.p.row_resid = v.d_res16;
    a.p.eps_rows = v.eps16;
    a.p.q_resid = ix.d_q_resid;
    a.p.kprime = kp;
    a.p.thr_global = ix.d_thr;
    a.p.ws_keys = w.d_ws;
    // Like the exact path's pass 1: when pass 1 rarely certifies, it only has to give each query its
    // threshold T, and every 4th tile of its lists gives a valid one (the rule lives in
    // ivf_finish_tc).
    // a tuned plan may fix the stride; at k ≥ 64 the rules start sampled (a full pass 1 then carries
    // the largest heaps and almost never certifies)
    const uint32_t stride = ix.forced_stride ? ix.forced_stride : (k >= 64 ? ivf_sampled_stride() : w.tc_stride);
    a.p.tile_stride = stride;
    a.p.heap_k = stride > 1 ? std::max(1u, std::min(kp, k)) : kp;  // a sampled pass 1 only yields T
    a.p.it_item_off = w.d_item_off;
    a.p.it_item_list = w.d_item_list;
    a.p.it_list_cnt = w.d_list_cnt;
    a.p.it_offsets = v.d_offsets;
    a.p.it_qblock_off = w.d_qblock_off;
    a.p.it_lane_qid = w.d_lane_qid;
    a.p.it_lane_slot = w.d_lane_slot;
    a.p.row_map = v.d_row_map;
    a.p.it_nlist = nlist;
    a.p.it_chunk_rows = kChunkRows;
    a.p.it_next = w.d_counters + 8;  // the CTAs take items from this counter
    cudaEvent_t ev_a = nullptr;
    ix.scan_event_begin(s, ev_a);
    e = launch_scan_tc(a, false, 0, s);
    ix.scan_event_end(s, ev_a);
    if (e != cudaSuccess) return cuda_error(e, "IVF tensor-core scan launch");
    uint32_t p2 = 1;
    while (p2 < kp) p2 <<= 1;
    ivf_merge_kernel<<<nq, 512, p2 * sizeof(uint64_t), s>>>(w.d_ws, w.d_q_slot_off, kp, ix.d_cand_idx, ix.d_cand_sim,
                                                            ix.d_cand_cnt);
    count_launch();
    RerankArgs r;
    r.base = v.d_reordered;  // the slot keys hold list positions
    r.row_map = v.d_row_map;
    r.ds = static_cast<uint32_t>(ix.ds);
    r.queries = ix.d_qn;
    r.cand_idx = ix.d_cand_idx;
    r.cand_sim = ix.d_cand_sim;
    r.cand_cnt = ix.d_cand_cnt;
    r.nq = nq;
    r.kp = kp;
    r.k = k;
    r.idx_out = o_idx;
    r.sim_out = o_sim;
    r.cnt_out = o_cnt;
    r.cert_out = ix.d_cert;
    r.kth_out = ix.d_kth;
    r.certify = stride == 1;
    if ((e = launch_rerank(r, s)) != cudaSuccess) return cuda_error(e, "rerank launch");

    // ---- pass 2: every probed row whose bound reaches T, for the uncertified queries ----
    uint32_t* d_m = ix.d_fbn + 1;     // uncertified queries
    uint32_t* d_fail = ix.d_fbn + 2;  // of them, collections that overflowed
    launch_compact_zero_flags(ix.d_cert, nq, ix.d_ids, d_m, s);
    ivf_pass2_thr_kernel<<<(nq + 255) / 256, 256, 0, s>>>(ix.d_cert, ix.d_kth, nq, ix.d_q2_thr);
    count_launch();
    cudaMemsetAsync(ix.d_cnt2, 0, nq * sizeof(uint32_t), s);
    a.stages = plan2.stages;
    a.stream_a = plan2.stream_a;
    a.p.tile_stride = 1;
    a.p.kprime = 0;
    a.p.q_thr = ix.d_q2_thr;
    a.p.cand_rows = ix.d_rows2;
    a.p.cand_cnt = ix.d_cnt2;
    a.p.cap2 = cap2;
    a.p.live_q = d_m;  // item mode: the whole pass returns at once when every query certified
    a.p.it_next = w.d_counters + 9;
    ix.scan_event_begin(s, ev_a);
    e = launch_scan_tc(a, false, 1, s);
    ix.scan_event_end(s, ev_a);
    if (e != cudaSuccess) return cuda_error(e, "IVF tensor-core scan launch (pass 2)");
    e = launch_rerank_collected(v.d_reordered, static_cast<uint32_t>(ix.ds), ix.d_qn, ix.d_ids, nq, ix.d_rows2,
                                ix.d_cnt2, cap2, k, ix.d_q2_thr, ix.d_rslots, o_idx, o_sim, o_cnt, ix.d_ok2, s, true,
                                d_m, v.d_row_map);
    if (e != cudaSuccess) return cuda_error(e, "rerank launch (pass 2)");
    launch_compact_zero_flags(ix.d_ok2, nq, ix.d_tcfail, d_fail, s, d_m);
    // the plan's totals and the pass counts come back with the results
    cudaMemcpyAsync(w.h_probed, w.d_counters, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(ix.h_fbn, ix.d_fbn, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    ix.last_tc_n = nq;
    ix.stats.kernel_launches += 14;
    ix.stats.path = 5;
    ix.stats.nprobe = np;
    ix.stats.rerank_width = kp;
    ix.stats.pass1_tile_stride = stride;
    return NNDEX_OK;
}

// After the stream has completed an ivf_search_tc batch: statistics, the pass-1 stride rule, and
// the FP32 list scan for queries whose collection overflowed (outputs patched in place; it
// synchronises the stream again only then).
int ivf_finish_tc(CudaIndex& ix, uint32_t nq, uint32_t k, uint64_t* o_idx, float* o_sim, uint32_t* o_cnt,
                  cudaStream_t s) {
    IvfScratch& w = ix.ivf_scratch;
    const uint32_t m = ix.h_fbn[1], failed_n = ix.h_fbn[2];
    ix.stats.rows_scanned = w.h_probed[3];
    ix.stats.ivf_rows_streamed = w.h_probed[4];
    ix.stats.ivf_rows_union = w.h_probed[5];
    ix.stats.certified = m == 0 ? 1u : 0u;
    ix.stats.second_pass_queries = m;
    ix.stats.fp32_fallback_queries = failed_n;
    int st;
    if (m) {
        // rows collected by pass 2 (the counts of the uncertified queries, read after the batch)
        if ((st = grow_pinned(ix.h_ok2, ix.cap_hok2, nq, "pinned buffer"))) return st;
        if ((st = grow_pinned(ix.h_ids, ix.cap_hids, nq, "pinned buffer"))) return st;
        cudaMemcpyAsync(ix.h_ok2, ix.d_cnt2, nq * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(ix.h_ids, ix.d_cert, nq * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        const cudaError_t e0 = cudaStreamSynchronize(s);
        if (e0 != cudaSuccess) return cuda_error(e0, "IVF search");
        uint64_t total = 0;
        for (uint32_t i = 0; i < nq; ++i)
            if (!ix.h_ids[i]) total += std::min<uint32_t>(ix.h_ok2[i], kSecondPassCap);
        ix.stats.pass2_rows += total;
    }
    // the rule learns from batches that ran its own stride (a full pass 1 that certified few)
    if (!ix.forced_stride && w.tc_stride == 1 && ix.stats.pass1_tile_stride == 1 && m * 2 > nq) {
        w.tc_stride = ivf_sampled_stride();
        ix.drop_graphs();  // a captured batch keeps its stride
    }
    if (failed_n == 0) return NNDEX_OK;
    // ---- FP32 list scan for the queries whose collection overflowed ----
    if ((st = grow_pinned(ix.h_ids, ix.cap_hids, nq, "pinned buffer"))) return st;
    if ((st = grow_pinned(ix.h_ok2, ix.cap_hok2, nq, "pinned buffer"))) return st;
    cudaMemcpyAsync(ix.h_ids, ix.d_ids, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(ix.h_ok2, ix.d_tcfail, failed_n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaError_t e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "IVF search");
    std::vector<uint32_t> failed(failed_n);
    for (uint32_t i = 0; i < failed_n; ++i) failed[i] = ix.h_ids[ix.h_ok2[i]];
    const uint32_t mf = failed_n;
    if ((st = grow(ix.d_qsub, ix.cap_qsub, static_cast<size_t>(mf) * ix.ds, "fallback buffer"))) return st;
    for (uint32_t i = 0; i < mf; ++i)
        cudaMemcpyAsync(ix.d_qsub + static_cast<uint64_t>(i) * ix.ds, ix.d_qn + static_cast<uint64_t>(failed[i]) * ix.ds,
                        ix.ds * sizeof(float), cudaMemcpyDeviceToDevice, s);
    if ((st = grow(ix.d_fb_idx, ix.cap_fb_idx, static_cast<size_t>(mf) * k, "fallback buffer"))) return st;
    if ((st = grow(ix.d_fb_sim, ix.cap_fb_sim, static_cast<size_t>(mf) * k, "fallback buffer"))) return st;
    if ((st = grow(ix.d_fb_cnt, ix.cap_fb_cnt, mf, "fallback buffer"))) return st;
    const nndex_cuda_search_stats keep = ix.stats;
    if ((st = ivf_search(ix, ix.d_qsub, mf, k, ix.d_fb_idx, ix.d_fb_sim, ix.d_fb_cnt, s))) return st;
    ix.stats = keep;
    for (uint32_t i = 0; i < mf; ++i) {
        const uint64_t q = failed[i];
        cudaMemcpyAsync(o_idx + q * k, ix.d_fb_idx + static_cast<uint64_t>(i) * k, k * sizeof(uint64_t),
                        cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(o_sim + q * k, ix.d_fb_sim + static_cast<uint64_t>(i) * k, k * sizeof(float),
                        cudaMemcpyDeviceToDevice, s);
        if (o_cnt) cudaMemcpyAsync(o_cnt + q, ix.d_fb_cnt + i, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    }
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "IVF search");
    return NNDEX_OK;
}

}  // namespace nndex
