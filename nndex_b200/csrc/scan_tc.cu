// scan_tc.cu — K3: tensor-core (tcgen05) scan of the BF16 / FP8-E4M3 base, and K4: exact FP32 rerank.
//
// This is the large-batch path of nndex's exact search (the reference's GEMM strategies,
// src/cpu.rs:256-341): S = Q̂·X̂ᵀ on the 5th-generation tensor cores with FP32 accumulation in TMEM.
// Scores never reach HBM. The result is the exact FP32 top-k, proven per query:
//
//   Every row r gets an upper bound of its exact score from its approximate score:
//       s_r ≤ u_r = s̃_r + ‖δx_r‖(1 + ‖δq‖) + ‖δq‖ + ε_acc
//   (q·x − q̂·x̂ = q·δx + δq·x̂, ‖q‖ = 1, Cauchy–Schwarz; ε_acc bounds the FP32 accumulation).
//   Pass 1 (kMode 0) keeps, per query, the k′ rows with the largest u_r (a min-heap per query in
//   shared memory, thresholds shared across CTAs through a global per-query key). K4 re-scores the
//   k′ candidates exactly in FP32; the exact k-th score T is a lower bound of the true k-th score.
//   If T > the k′-th upper bound, no other row can enter the top-k: the query is done.
//   Pass 2 (kMode 1), for the other queries only: collect every row with u_r ≥ T (no row with
//   u_r < T can reach the top-k, since k rows already score ≥ T), and re-score them exactly.
//   Only a query whose pass-2 set overflows its buffer is re-run on the FP32 scan.
//
// K3 layout. One CTA = 128 queries (one TMEM lane each; the query block is the MMA's A operand,
// resident in shared memory) × one range of base rows. Warp 0 issues TMA loads of 256-row base
// tiles, one 128-byte K slab per ring stage (128 B swizzle); warp 1 issues tcgen05.mma (M = 128,
// N = 256, 4 instructions per slab) into one of two 256-column FP32 accumulators in TMEM; warps 2-5
// read the finished accumulator with tcgen05.ld (each thread: one query's 256 scores, in 32-column
// chunks, loads double-buffered), reject almost every score with one compare against
// (threshold − largest possible bound slack), and bound/insert the rare survivors. Base tiles stay
// in L2 for the other query blocks of the same row range. No TMA multicast.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>

#include "common.cuh"
#include "internal.h"
#include "select.cuh"
#include "tc.cuh"

namespace nndex {

namespace {
constexpr int kM = 128;               // queries per CTA (TMEM lanes)
constexpr int kN = 256;               // base rows per tile (MMA N)
constexpr uint32_t kAChunk = kM * 128;
constexpr uint32_t kBChunk = kN * 128;
// Warps: 0 TMA, 1 MMA, then the epilogue: 4 warps in pass 1 (one thread owns a query's heap), 8 in
// pass 2 (two warps per TMEM lane quarter, each reading half of the tile's columns: collection has
// no per-query state beyond the threshold, and the epilogue, not the MMA, bounds the pass).
template <int kMode>
constexpr uint32_t epi_warps() { return kMode == 1 ? 8u : 4u; }
// Pass 2: rows that pass the cut are staged per epilogue thread and appended to the query's
// collection kPass2Stage at a time (one atomic per group instead of one per row).
constexpr uint32_t kPass2Stage = 16;
template <int kMode>
constexpr int tc_threads() { return 64 + 32 * static_cast<int>(epi_warps<kMode>()); }
constexpr uint32_t kTmemCols = 512;   // two 256-column FP32 accumulators

NNDEX_DEVICE_INLINE uint8_t* align_1024(uint8_t* p) {
    const uint32_t a = smem_u32(p);
    return p + ((1024u - (a & 1023u)) & 1023u);
}

// tcgen05.wait::ld that also ties the 32 registers of the completed load, so no use of them can be
// scheduled before the wait.
NNDEX_DEVICE_INLINE void tmem_wait_ld_regs(uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.wait::ld.sync.aligned;"
        : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
          "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]), "+r"(v[15]),
          "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]), "+r"(v[22]), "+r"(v[23]),
          "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]), "+r"(v[29]), "+r"(v[30]), "+r"(v[31])
        :
        : "memory");
}

NNDEX_DEVICE_INLINE float pick(const uint32_t (&v)[32], uint32_t j) {
    uint32_t r = 0;
#pragma unroll
    for (uint32_t jj = 0; jj < 32; ++jj) r = (jj == j) ? v[jj] : r;
    return __uint_as_float(r);
}
}  // namespace

size_t tc_smem_bytes(uint32_t nchunks, uint32_t kprime, uint32_t stages, bool fp8, bool stream_a, uint32_t qb) {
    // qb: 1 = one resident query block and 256-row stages, 2 = two blocks and 128-row stages,
    // 3 = one block per CTA of a CTA pair and 128-row stages (the pair's tile is 256 rows)
    const size_t a_blocks = qb == 2 ? 2 : 1, stage_b = qb == 1 ? kBChunk : kBChunk / 2;
    size_t b = 1024;
    b += stream_a ? static_cast<size_t>(stages) * (kAChunk + kBChunk)
                  : a_blocks * nchunks * kAChunk + static_cast<size_t>(stages) * stage_b;
    b += static_cast<size_t>(kprime) * kM * 8;
    if (kprime == 0) b += static_cast<size_t>(kPass2Stage) * 8 * 32 * 4;  // pass 2: survivor staging
    b += (2 * stages + 10) * 8 + 16;
    return b;
}

uint32_t tc_stages_for(uint32_t nchunks, uint32_t kprime, bool fp8, bool stream_a, size_t smem_limit) {
    for (uint32_t st = 4; st >= 2; --st)
        if (tc_smem_bytes(nchunks, kprime, st, fp8, stream_a) <= smem_limit) return st;
    return 0;
}

uint32_t tc_pair_stages_for(uint32_t nchunks, bool fp8, size_t smem_limit) {
    for (uint32_t st = 5; st >= 4; --st)
        if (tc_smem_bytes(nchunks, 0, st, fp8, false, 2) <= smem_limit) return st;
    return 0;
}

uint32_t tc_cta_pair_stages_for(uint32_t nchunks, bool fp8, size_t smem_limit) {
    for (uint32_t st : {8u, 6u})
        if (tc_smem_bytes(nchunks, 0, st, fp8, false, 3) <= smem_limit) return st;
    return 0;
}

// Per-query epilogue state.
struct EpiState {
    uint32_t n;                  // heap size (pass 1)
    unsigned long long thr_key;  // pass 1: key a candidate must beat
    float thr_f;                 // pass 1: score of thr_key; pass 2: T
    float cut;                   // thr_f − largest bound slack: scores below cannot survive
};

// A score that passed the cheap filter: apply its exact bound, then insert (pass 1) or collect
// (pass 2).
template <int kMode>
NNDEX_DEVICE_INLINE void epi_survivor(const TcParams& p, EpiState& st, uint64_t* heap, uint32_t lrow, uint32_t q,
                                      float u, uint64_t row, float slack) {
    if (u < st.thr_f) return;
    if (kMode == 0) {
        const uint64_t key = make_key(u, static_cast<uint32_t>(row));
        if (key <= st.thr_key) return;
        const uint32_t kp = p.heap_k;
        if (st.n < kp) {
            uint32_t i = st.n++;
            while (i > 0) {
                const uint32_t pp = (i - 1) >> 1;
                const uint64_t hp = heap[pp * kM + lrow];
                if (hp <= key) break;
                heap[i * kM + lrow] = hp;
                i = pp;
            }
            heap[i * kM + lrow] = key;
        } else {
            uint32_t i = 0;
            for (;;) {
                const uint32_t l = 2 * i + 1;
                if (l >= st.n) break;
                const uint32_t r = l + 1;
                uint64_t hm = heap[l * kM + lrow];
                uint32_t m = l;
                if (r < st.n) {
                    const uint64_t hr = heap[r * kM + lrow];
                    if (hr < hm) {
                        hm = hr;
                        m = r;
                    }
                }
                if (hm >= key) break;
                heap[i * kM + lrow] = hm;
                i = m;
            }
            heap[i * kM + lrow] = key;
        }
        if (st.n == kp) {
            const uint64_t mn = heap[lrow];
            if (mn > st.thr_key) {
                st.thr_key = mn;
                st.thr_f = key_score(mn);
                st.cut = st.thr_f - slack;
            }
        }
    } else {
        const uint32_t pos = atomicAdd(&p.cand_cnt[q], 1u);
        if (pos < p.cap2) p.cand_rows[static_cast<size_t>(q) * p.cap2 + pos] = static_cast<uint32_t>(row);
    }
}

// kStreamA: the query block's K slabs are not resident; each ring stage carries the matching query
// slab beside the base slab (re-read from L2 per tile). It frees nchunks × 16 KB of shared memory
// for the pass-1 heaps, which large D × large k needs (D = 512, k = 100: 128 KB of queries).
// kItems: the IVF list scan (TcParams' item fields): the CTA's queries are a gathered block of the
// queries probing one list and its rows one chunk of that list's reordered rows; keys and collected
// rows carry original row indices, and pass-1 heaps go to the (query, chunk) output slots.
// kQB = 2 (pass 2 only): two resident query blocks per CTA (256 queries) against 128-row base tiles.
// Each slab of a base tile feeds two MMAs (M = 128, N = 128), one per block, into the two halves of
// the 256-column accumulator, so a CTA reads half the base bytes per FLOP: the pass is otherwise
// bound by how fast L2 feeds the base tiles (1 byte per 128 FLOPs). The tile map's box is 128 rows.
// kPair (pass 2 only): CTA pairs (a cluster of two) share each 256-row base tile: each CTA loads
// its own query block and 128 of the tile's rows, and the even CTA issues M = 256, N = 256 MMAs
// (cta_group::2) over both CTAs' shared memory into both CTAs' TMEM, so each SM reads half the base
// bytes per FLOP at the full MMA shape. The barriers that gate MMAs (slabs landed, query blocks
// landed, accumulators drained) are the even CTA's, armed for both CTAs' bytes and arrivals; the
// MMA completions arrive on both CTAs' barriers (slab free, accumulator ready). The tile map's box
// is 128 rows.
template <bool kFp8, int kST, int kMode, bool kStreamA, bool kItems, int kQB, bool kPair = false>
__global__ void __launch_bounds__(tc_threads<kMode>(), 1)
    scan_tc_kernel(const __grid_constant__ CUtensorMap tmap_q, const __grid_constant__ CUtensorMap tmap_b,
                   const TcParams p) {
    static_assert(kQB == 1 || (kQB == 2 && kMode == 1 && !kStreamA && !kItems), "two query blocks: pass 2 only");
    static_assert(!kPair || (kQB == 1 && kMode == 1 && !kStreamA && !kItems), "CTA pairs: pass 2 only");
    constexpr uint32_t kNT = kQB == 2 ? kN / 2 : kN;  // base rows per tile (MMA N)
    constexpr uint32_t kLoadRows = kPair ? kN / 2 : kNT;  // base rows per tile this CTA loads
    constexpr uint32_t kQC = kM * kQB;                // queries per CTA
    constexpr uint32_t kElems = kFp8 ? 128 : 64;      // K elements per 128-byte slab
    constexpr uint32_t kStage = kStreamA ? kAChunk + kBChunk : kLoadRows * 128;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = align_1024(smem_raw);
    uint8_t* a_smem = smem;  // resident query slabs (kStreamA: none), block-major
    uint8_t* b_smem = a_smem + (kStreamA ? 0 : static_cast<size_t>(kQB) * p.nchunks * kAChunk);
    uint64_t* heap = reinterpret_cast<uint64_t*>(b_smem + static_cast<size_t>(kST) * kStage);
    uint32_t* stage2 = reinterpret_cast<uint32_t*>(heap + static_cast<size_t>(p.kprime) * kM);  // pass 2
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(stage2 + (kMode == 1 ? kPass2Stage * 8 * 32 : 0));
    uint64_t* empty_bar = full_bar + kST;
    uint64_t* a_full = empty_bar + kST;
    uint64_t* a_free = a_full + 1;  // item mode: the MMAs of the last item have read its query block
    uint64_t* wfull = a_free + 1;   // item mode: the next item's id is in witem[slot]
    uint64_t* wempty = wfull + 2;   // item mode: the MMA and epilogue warps have read witem[slot]
    uint64_t* tfull = wempty + 2;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    volatile uint32_t* abort_flag = tmem_slot + 1;
    volatile uint32_t* witem = tmem_slot + 2;  // [2]

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t rank = kPair ? cluster_ctarank() : 0u;  // the CTA's place in its pair
    const bool leader = rank == 0;                          // pairs: the even CTA issues the MMAs
    uint32_t grid_q0 = blockIdx.x * kQC;
    uint32_t range = blockIdx.y, nranges = gridDim.y;
    uint64_t range_rows = p.range_rows;
    uint32_t nq_live = p.nq;
    if (!kItems && p.live_q) {
        // The device count decides the grid's shape (tc_range_split, as the host splits pass 1);
        // CTAs past the work items return before any set-up.
        nq_live = *p.live_q;
        const uint64_t nqb = (nq_live + kQC - 1) / kQC;
        if (nqb == 0) return;
        uint64_t nr = 0;
        tc_range_split(p.rows, kPair ? (nqb + 1) / 2 * 2 : nqb, p.sm_count, nr, range_rows);
        if (kPair) {
            // pairs of query blocks (the last one may have no queries: its CTA still loads its half
            // of the base tiles); both CTAs of a pair return here, or neither
            const uint64_t npairs = (nqb + 1) / 2, pair = blockIdx.x >> 1;
            if (pair >= npairs * nr) return;
            grid_q0 = static_cast<uint32_t>((pair % npairs) * 2 + rank) * kQC;
            range = static_cast<uint32_t>(pair / npairs);
        } else {
            if (blockIdx.x >= nqb * nr) return;
            // consecutive CTAs take the query blocks of one row range, as the 2-D grid orders them:
            // the CTAs resident together read the same base tiles, which then come from L2 after
            // the first
            grid_q0 = static_cast<uint32_t>(blockIdx.x % nqb) * kQC;
            range = static_cast<uint32_t>(blockIdx.x / nqb);
        }
        nranges = static_cast<uint32_t>(nr);
    }
    // The CTA's work: one (query block, row range) in the grid modes. In item mode its producer
    // thread takes up to kItemsPerCta of the plan's items (each a chunk of one list × one gathered
    // query block) from a global counter and hands each item's id to the MMA and epilogue warps
    // through two shared-memory slots; TMEM, barriers and the base ring stay across them, so the
    // next item's base tiles stream while the last one's epilogue drains. (With one CTA per SM
    // taking every item, the kernel held all SMs until its last item and other streams' kernels
    // waited behind it.)
    constexpr uint32_t kNoItem = 0xFFFFFFFFu;
    constexpr uint32_t kItemsPerCta = 4;
    uint32_t total = 0;
    if (kItems) {
        total = p.it_item_off[p.it_nlist];
        // pass 2 has nothing to do when every query certified (the device count of the others is 0)
        if (kMode == 1 && p.live_q && *p.live_q == 0) return;
        if (total == 0) return;
    }
    const uint64_t tile_step = static_cast<uint64_t>(kNT) * p.tile_stride;
    struct Work {
        uint32_t q0, chunk, ntiles, nblk;
        uint64_t row_begin, row_end;
    };
    auto work_of = [&](uint32_t wi) {
        Work w;
        w.chunk = 0;  // item mode: the chunk of the list (its output slot offset)
        if (kItems) {
            const uint32_t lo = p.it_item_list[wi];  // the item's list
            const uint32_t groups = (p.it_list_cnt[lo] + kM - 1) / kM;
            const uint32_t local = wi - p.it_item_off[lo];
            w.chunk = local / groups;
            w.q0 = (p.it_qblock_off[lo] + local % groups) * kM;
            w.row_begin = p.it_offsets[lo] + static_cast<uint64_t>(w.chunk) * p.it_chunk_rows;
            const uint64_t le = p.it_offsets[lo + 1];
            w.row_end = (w.row_begin + p.it_chunk_rows) < le ? (w.row_begin + p.it_chunk_rows) : le;
        } else {
            w.q0 = grid_q0;
            w.row_begin = static_cast<uint64_t>(range) * range_rows;
            w.row_end = (w.row_begin + range_rows) < p.rows ? (w.row_begin + range_rows) : p.rows;
        }
        // query blocks with at least one query: a second block past the last query is neither
        // loaded nor multiplied (its epilogue lanes have no query)
        w.nblk = (kQB == 2 && w.q0 + kM >= nq_live) ? 1u : static_cast<uint32_t>(kQB);
        w.ntiles = w.row_end > w.row_begin
                       ? static_cast<uint32_t>((w.row_end - w.row_begin + tile_step - 1) / tile_step)
                       : 0u;
        return w;
    };
    const uint32_t nchunks = p.nchunks;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kST; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(a_full, 1);
        mbar_init(a_free, 1);
        for (int b = 0; b < 2; ++b) {
            mbar_init(&wfull[b], 1);
            mbar_init(&wempty[b], 1 + epi_warps<kMode>());
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], (kPair ? 2 : 1) * epi_warps<kMode>());  // pairs: both CTAs' epilogues
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        if constexpr (kPair) {
            tc::tmem_alloc_pair(tmem_slot, kTmemCols);
            tc::tmem_relinquish_pair();
        } else {
            tc::tmem_alloc(tmem_slot, kTmemCols);
            tc::tmem_relinquish();
        }
    }
    tc::fence_before_sync();
    // pairs: the other CTA's barriers are initialised before any copy or arrival reaches them
    if (kPair) cluster_sync_all();
    else __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            tma_prefetch_desc(&tmap_q);
            tma_prefetch_desc(&tmap_b);
            // Base tiles are read by every query block of the same row range at about the same
            // time: keep them in L2 with the default policy (no evict-first hint).
            uint32_t it = 0, a_loads = 0;
            bool stop = false;
            for (uint32_t j = 0; !stop; ++j) {
                uint32_t wi = 0;
                if (kItems) {
                    // take the next item; its slot is free once both readers took the item before
                    const uint32_t slot = j & 1u;
                    if (j >= 2 && !mbar_wait_bounded(&wempty[slot], ((j >> 1) - 1) & 1u, kWaitBudgetCycles)) {
                        *abort_flag = 1;
                        record_status(p.status, kStatusTimeout);
                        break;
                    }
                    const unsigned long long g = j < kItemsPerCta ? atomicAdd(p.it_next, 1ull) : ~0ull;
                    wi = g < total ? static_cast<uint32_t>(g) : kNoItem;
                    witem[slot] = wi;
                    mbar_arrive(&wfull[slot]);
                    if (wi == kNoItem) break;
                } else if (j > 0) {
                    break;
                }
                const Work w = work_of(wi);
                if (!kStreamA) {
                    // the previous item's MMAs have read its query block (a_free) before this one's
                    // replaces it
                    if (j > 0 && !mbar_wait_bounded(a_free, (j - 1) & 1u, kWaitBudgetCycles)) {
                        *abort_flag = 1;
                        record_status(p.status, kStatusTimeout);
                        stop = true;
                        break;
                    }
                    if constexpr (kPair) {
                        // both CTAs' query blocks complete on the even CTA's barrier
                        if (leader) mbar_arrive_expect_tx(a_full, 2u * nchunks * kAChunk);
                        const uint32_t a_bar = cluster_map(a_full, 0);
                        for (uint32_t c = 0; c < nchunks; ++c)
                            tma_load_2d_pair(a_smem + static_cast<size_t>(c) * kAChunk, &tmap_q, a_bar,
                                             static_cast<int32_t>(c * kElems), static_cast<int32_t>(w.q0));
                    } else {
                        mbar_arrive_expect_tx(a_full, w.nblk * nchunks * kAChunk);
                        for (uint32_t b = 0; b < w.nblk; ++b)
                            for (uint32_t c = 0; c < nchunks; ++c)
                                tma_load_2d(a_smem + static_cast<size_t>(b * nchunks + c) * kAChunk, &tmap_q,
                                            a_full, static_cast<int32_t>(c * kElems),
                                            static_cast<int32_t>(w.q0 + b * kM));
                    }
                    ++a_loads;
                }
                for (uint32_t t = 0; t < w.ntiles && !stop; ++t) {
                    const int32_t y = static_cast<int32_t>(w.row_begin + static_cast<uint64_t>(t) * tile_step);
                    for (uint32_t c = 0; c < nchunks; ++c) {
                        const uint32_t s = it % kST, u = it / kST;
                        if (u > 0 && !mbar_wait_bounded(&empty_bar[s], (u - 1) & 1u, kWaitBudgetCycles)) {
                            *abort_flag = 1;
                            record_status(p.status, kStatusTimeout);
                            stop = true;
                            break;
                        }
                        if (*abort_flag) {
                            stop = true;
                            break;
                        }
                        uint8_t* stage = b_smem + static_cast<size_t>(s) * kStage;
                        if constexpr (kPair) {
                            // this CTA's 128 rows of the pair's 256-row tile; both halves complete on
                            // the even CTA's barrier, which expects both
                            if (leader) mbar_arrive_expect_tx(&full_bar[s], 2u * kStage);
                            tma_load_2d_pair(stage, &tmap_b, cluster_map(&full_bar[s], 0),
                                             static_cast<int32_t>(c * kElems),
                                             y + static_cast<int32_t>(rank * kLoadRows));
                        } else {
                            mbar_arrive_expect_tx(&full_bar[s], kStage);
                            if (kStreamA)
                                tma_load_2d(stage + kBChunk, &tmap_q, &full_bar[s], static_cast<int32_t>(c * kElems),
                                            static_cast<int32_t>(w.q0));
                            tma_load_2d(stage, &tmap_b, &full_bar[s], static_cast<int32_t>(c * kElems), y);
                        }
                        ++it;
                    }
                }
            }
            // Drain every copy this thread issued before the CTA may exit. (Pairs: the odd CTA's copies
            // complete on the even CTA's barriers, which the even CTA drains; neither CTA leaves the
            // closing cluster barrier before the other reaches it.)
            if (!kStreamA && a_loads > 0 && leader &&
                !mbar_wait_bounded(a_full, (a_loads - 1) & 1u, kWaitBudgetCycles))
                record_status(p.status, kStatusTimeout);
            const uint32_t used = !leader ? 0u : (it < static_cast<uint32_t>(kST) ? it : kST);
            for (uint32_t s = 0; s < used; ++s) {
                const uint32_t uses = (it - s + kST - 1) / kST;
                if (!mbar_wait_bounded(&full_bar[s], (uses - 1) & 1u, kWaitBudgetCycles))
                    record_status(p.status, kStatusTimeout);
            }
            if (kPair) {
                // the even CTA's MMA completions also arrive on this CTA's slab barriers: wait for the
                // last one of every slab before the CTA may leave
                const uint32_t used_e = it < static_cast<uint32_t>(kST) ? it : kST;
                for (uint32_t s = 0; s < used_e; ++s) {
                    const uint32_t uses = (it - s + kST - 1) / kST;
                    if (!mbar_wait_bounded(&empty_bar[s], (uses - 1) & 1u, kWaitBudgetCycles))
                        record_status(p.status, kStatusTimeout);
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer (pairs: the even CTA's, for both) ----------------
        if (lane == 0 && leader) {
            constexpr uint32_t idesc = tc::instr_desc<kFp8, kPair ? 2 * kM : kM, kNT>();
            const uint32_t a_addr0 = smem_u32(a_smem), b_addr0 = smem_u32(b_smem);
            uint32_t it = 0, tg = 0;  // slabs and tiles over all of the CTA's work
            for (uint32_t j = 0;; ++j) {
                uint32_t wi = 0;
                if (kItems) {
                    const uint32_t slot = j & 1u;
                    if (*abort_flag || !mbar_wait_bounded(&wfull[slot], (j >> 1) & 1u, kWaitBudgetCycles)) {
                        if (!*abort_flag) {
                            *abort_flag = 1;
                            record_status(p.status, kStatusTimeout);
                        }
                        break;
                    }
                    wi = witem[slot];
                    mbar_arrive(&wempty[slot]);
                    if (wi == kNoItem) break;
                    // another item: the previous one's MMAs are all issued, and its query block may
                    // be replaced once they complete (never committed after the CTA's last item,
                    // which nothing waits for)
                    if (!kStreamA && j > 0) tc::commit(a_free);
                } else if (j > 0) {
                    break;
                }
                const Work w = work_of(wi);
                if (!kStreamA && !*abort_flag && !mbar_wait_bounded(a_full, j & 1u, kWaitBudgetCycles)) {
                    *abort_flag = 1;
                    record_status(p.status, kStatusTimeout);
                }
                tc::fence_after_sync();
                for (uint32_t t = 0; t < w.ntiles; ++t, ++tg) {
                    const uint32_t buf = tg & 1u, ub = tg >> 1;
                    if (ub > 0 && !*abort_flag &&
                        !mbar_wait_bounded(&tempty[buf], (ub - 1) & 1u, kWaitBudgetCycles)) {
                        *abort_flag = 1;
                        record_status(p.status, kStatusTimeout);
                    }
                    tc::fence_after_sync();
                    const uint32_t d = tmem_base + buf * kN;  // kQB = 2: block b in columns [b·128, b·128 + 128)
                    for (uint32_t c = 0; c < nchunks; ++c, ++it) {
                        const uint32_t s = it % kST, u = it / kST;
                        if (!*abort_flag && !mbar_wait_bounded(&full_bar[s], u & 1u, kWaitBudgetCycles)) {
                            *abort_flag = 1;
                            record_status(p.status, kStatusTimeout);
                        }
                        tc::fence_after_sync();
                        if (!*abort_flag) {
                            const uint32_t b_addr = b_addr0 + s * kStage;
                            for (uint32_t b = 0; b < w.nblk; ++b) {
                                const uint32_t a_addr =
                                    kStreamA ? b_addr + kBChunk : a_addr0 + (b * nchunks + c) * kAChunk;
#pragma unroll
                                for (uint32_t kk = 0; kk < 4; ++kk) {
                                    if constexpr (kPair)
                                        tc::mma_pair<kFp8>(d, tc::smem_desc_sw128(a_addr + kk * 32),
                                                           tc::smem_desc_sw128(b_addr + kk * 32), idesc,
                                                           (c | kk) != 0u ? 1u : 0u);
                                    else
                                        tc::mma<kFp8>(d + b * kNT, tc::smem_desc_sw128(a_addr + kk * 32),
                                                      tc::smem_desc_sw128(b_addr + kk * 32), idesc,
                                                      (c | kk) != 0u ? 1u : 0u);
                                }
                            }
                        }
                        // frees the slab (pairs: in both CTAs) once the MMAs above have read it
                        if constexpr (kPair) tc::commit_pair(&empty_bar[s], 0x3);
                        else tc::commit(&empty_bar[s]);
                    }
                    // the accumulator is complete (pairs: both CTAs' halves)
                    if constexpr (kPair) tc::commit_pair(&tfull[buf], 0x3);
                    else tc::commit(&tfull[buf]);
                }
            }
        }
    } else {
        // ---------------- epilogue: one query per thread (pass 2: two threads, half a tile each) ----
        constexpr uint32_t kEpiW = epi_warps<kMode>();
        constexpr uint32_t kWPB = kEpiW / 4 / kQB;            // warps per (TMEM lane quarter, query block)
        constexpr uint32_t kChunks = (kNT / 32) / kWPB;       // 32-column chunks per thread
        const uint32_t ew = warp - 2;
        const uint32_t blk = (ew / 4) / kWPB;                 // the thread's query block
        const uint32_t c_begin = ((ew / 4) % kWPB) * kChunks;
        const uint32_t quarter = warp & 3u;
        const uint32_t lrow = quarter * 32 + lane;
        // pass 2: this thread's staged rows and its append of them to the query's collection
        uint32_t* my_stage = stage2 + (ew * 32 + lane) * kPass2Stage;
        const uint32_t taddr0 = tmem_base + ((quarter * 32u) << 16);
        const bool per_row_bound = p.tile_stride == 1;
        uint32_t tg = 0;  // tiles over all of the CTA's work
        for (uint32_t jw = 0;; ++jw) {
            uint32_t wi = 0;
            if (kItems) {
                // lane 0 takes the item and the warp follows its decision (no lane leaves alone)
                const uint32_t slot = jw & 1u;
                uint32_t got = kNoItem;
                if (lane == 0) {
                    if (!*abort_flag && mbar_wait_bounded(&wfull[slot], (jw >> 1) & 1u, kWaitBudgetCycles)) {
                        got = witem[slot];
                        mbar_arrive(&wempty[slot]);
                    } else if (!*abort_flag) {
                        *abort_flag = 1;
                        record_status(p.status, kStatusTimeout);
                    }
                }
                wi = __shfl_sync(0xffffffffu, got, 0);
                if (wi == kNoItem) break;
            } else if (jw > 0) {
                break;
            }
            const Work w = work_of(wi);
            const uint32_t q0 = w.q0;
            const uint64_t row_begin = w.row_begin, row_end = w.row_end;
            const uint32_t q = kItems ? p.it_lane_qid[q0 + lrow] : q0 + blk * kM + lrow;
            const bool valid_q = kItems ? q != 0xFFFFFFFFu : q < nq_live;
            uint32_t staged = 0;
            auto flush_stage = [&]() {
                const uint32_t pos = atomicAdd(&p.cand_cnt[q], staged);
                for (uint32_t i = 0; i < staged; ++i)
                    if (pos + i < p.cap2) p.cand_rows[static_cast<size_t>(q) * p.cap2 + pos + i] = my_stage[i];
                staged = 0;
            };
            const float qs = (kFp8 && valid_q) ? p.q_scale[q] : 1.0f;
            const float rq = valid_q ? p.q_resid[q] : 0.0f;
            const float b_mul = 1.0f + rq, b_add = rq + p.eps_acc;
            const float slack = fmaf(p.eps_rows, b_mul, b_add);  // the largest u_r − s̃_r over all rows
            EpiState st;
            st.n = 0;
            if (kMode == 0) {
                st.thr_key = valid_q ? p.thr_global[q] : ~0ull;
                st.thr_f = !valid_q ? INFINITY : (st.thr_key ? key_score(st.thr_key) : -INFINITY);
            } else {
                st.thr_key = 0;
                st.thr_f = valid_q ? p.q_thr[q] : INFINITY;
            }
            st.cut = st.thr_f - slack;
            for (uint32_t t = 0; t < w.ntiles; ++t, ++tg) {
                const uint32_t buf = tg & 1u, ub = tg >> 1;
                const uint64_t tile_row0 = row_begin + static_cast<uint64_t>(t) * tile_step;
                // FP8: the extremes of the row scales over this tile's rows (computed once per index),
                // so no thread needs the tile's 256 scales unless a score may survive
                float smin = 0.0f, smax = 0.0f;
                const float* sc = kFp8 ? p.row_scale + tile_row0 : nullptr;
                if (kFp8) {
                    const float2 mm = p.tile_scale[tile_row0 / kN];  // a 128-row tile lies in one 256-row tile
                    smin = mm.x;
                    smax = mm.y;
                }
                if (!*abort_flag && !mbar_wait_bounded(&tfull[buf], ub & 1u, kWaitBudgetCycles)) {
                    *abort_flag = 1;
                    record_status(p.status, kStatusTimeout);
                }
                tc::fence_after_sync();
                if (kMode == 0 && (t & 3u) == 3u && valid_q) {
                    const unsigned long long g = p.thr_global[q];
                    if (g > st.thr_key) {
                        st.thr_key = g;
                        st.thr_f = key_score(g);
                        st.cut = st.thr_f - slack;
                    }
                }
                const uint32_t taddr = taddr0 + buf * kN + blk * kNT;
                uint32_t va[32], vb[32];
                __syncwarp();
                tc::tmem_ld32(taddr + c_begin * 32, va);
                tmem_wait_ld_regs(va);
                // The cut in the domain of the accumulator's raw scores. FP8 scores are scaled by the
                // row's and the query's scales (both positive): a score can reach the cut only if its
                // raw value reaches cut / (largest row scale · query scale) when cut ≥ 0, or cut /
                // (smallest row scale · query scale) when cut < 0; 2⁻²⁰ of slack covers the roundings
                // of both sides.
                float raw_cut = st.cut;
                if (kFp8) {
                    const float den = (st.cut >= 0.0f ? smax : smin) * qs;
                    raw_cut = (den > 0.0f) ? st.cut / den : -INFINITY;
                    raw_cut -= fabsf(raw_cut) * 9.5367431640625e-07f;
                    if (!(raw_cut == raw_cut)) raw_cut = -INFINITY;  // an infinite cut filters nothing here
                }
                auto process = [&](const uint32_t(&v)[32], uint32_t c) {
                    // A padding lane (no query: past nq, or an empty slot of a gathered block) scores
                    // whatever its query row holds, +inf included; it never survives, since its
                    // index would address past the per-query outputs.
                    if (!valid_q) return;
                    // Almost every group of 32 scores is rejected by its largest one (a 5-level tree).
                    float m16[16];
#pragma unroll
                    for (uint32_t j = 0; j < 16; ++j) m16[j] = fmaxf(__uint_as_float(v[j]), __uint_as_float(v[j + 16]));
#pragma unroll
                    for (uint32_t h = 8; h > 0; h >>= 1)
#pragma unroll
                        for (uint32_t j = 0; j < h; ++j) m16[j] = fmaxf(m16[j], m16[j + h]);
                    if (!(m16[0] >= raw_cut)) return;
                    uint32_t mask = 0;
#pragma unroll
                    for (uint32_t j = 0; j < 32; ++j) {
                        float s = __uint_as_float(v[j]);
                        if (kFp8) s = (s * sc[c * 32 + j]) * qs;
                        mask |= (s >= st.cut ? 1u : 0u) << j;
                    }
                    while (mask) {  // survivors are rare once a threshold exists
                        const uint32_t j = __ffs(mask) - 1;
                        mask &= mask - 1;
                        const uint64_t row = tile_row0 + c * 32 + j;
                        if (row >= row_end) continue;
                        if (kMode == 1) {
                            // pass 2 keeps every row that passed the cut (the largest bound slack over
                            // all rows: a superset of the rows whose own bound reaches T); in item mode
                            // the row is a reordered position, mapped to its row by the rerank
                            my_stage[staged++] = static_cast<uint32_t>(row);
                            if (staged == kPass2Stage) flush_stage();
                            continue;
                        }
                        float s = pick(v, j);
                        if (kFp8) s = (s * sc[c * 32 + j]) * qs;
                        // The row's own bound when pass 1 may certify (every tile scanned); a sampled
                        // pass 1 only yields T, and the largest slack spares a dependent load per
                        // survivor. In item mode the key holds the list position (the rerank maps it).
                        const float u = per_row_bound ? fmaf(p.row_resid[row], b_mul, s + b_add) : s + slack;
                        epi_survivor<kMode>(p, st, heap, lrow, q, u, row, slack);
                    }
                };
#pragma unroll
                for (uint32_t cc = 0; cc < kChunks; cc += 2) {
                    const uint32_t c = c_begin + cc;
                    // tcgen05.ld and tcgen05.wait::ld are .sync.aligned: the whole warp executes each
                    // one together. process() loops per lane over its survivors (one lane may take
                    // every row while the others take none), so the warp reconverges before each.
                    __syncwarp();
                    tc::tmem_ld32(taddr + (c + 1) * 32, vb);
                    process(va, c);
                    __syncwarp();
                    tmem_wait_ld_regs(vb);
                    if (cc + 2 < kChunks) tc::tmem_ld32(taddr + (c + 2) * 32, va);
                    process(vb, c + 1);
                    if (cc + 2 < kChunks) {
                        __syncwarp();
                        tmem_wait_ld_regs(va);
                    }
                }
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) {
                    if (kPair) mbar_arrive_cluster(cluster_map(&tempty[buf], 0));  // the MMA issuer's barrier
                    else mbar_arrive(&tempty[buf]);
                }
            }
            if (kMode == 1 && staged) flush_stage();
            if (kMode == 0 && valid_q) {
                uint64_t* dst = kItems ? p.ws_keys + static_cast<size_t>(p.it_lane_slot[q0 + lrow] + w.chunk) * p.kprime
                                       : p.ws_keys + (static_cast<size_t>(q) * nranges + range) * p.kprime;
                for (uint32_t i = 0; i < p.kprime; ++i) dst[i] = i < st.n ? heap[i * kM + lrow] : 0ull;
                if (st.n == p.heap_k) atomicMax(&p.thr_global[q], static_cast<unsigned long long>(heap[lrow]));
            }
        }
    }
    // ---------------- teardown: release TMEM ----------------
    tc::fence_before_sync();
    // pairs: both CTAs are done with each other's shared memory, barriers and TMEM
    if (kPair) cluster_sync_all();
    else __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc::fence_after_sync();
        if constexpr (kPair) tc::tmem_dealloc_pair(tmem_base, kTmemCols);
        else tc::tmem_dealloc(tmem_base, kTmemCols);
    }
}

// ------------------------------------------------------------------------------------------
// Exact FP32 dot product in the order of the FP32 scan (scan_fp32.cu): eight chains, one per
// 16-byte chunk position ch of each 128-byte slab, each accumulating its chunk's four products slab
// by slab with FMA; then ((c0+c1)+(c2+c3)) + ((c4+c5)+(c6+c7)). Called by 8 consecutive lanes (one
// per ch); every lane returns the full sum. So a query's scores are bit-identical on every path.
// ------------------------------------------------------------------------------------------
// The query is in shared memory (`ys`): kU of the row's slabs (a gather) are loaded before their
// FMAs, which stay in slab order.
template <uint32_t kU>
NNDEX_DEVICE_INLINE float dot_scan_order(const float* __restrict__ x, const float* ys, uint32_t nbox, uint32_t ch,
                                            bool live) {
    float acc = 0.0f;
    if (live) {
        const float* xa = x + ch * 4;
        const float* ya = ys + ch * 4;
        uint32_t bx = 0;
        for (; bx + kU <= nbox; bx += kU) {
            float4 a[kU];
#pragma unroll
            for (uint32_t u = 0; u < kU; ++u) a[u] = __ldg(reinterpret_cast<const float4*>(xa + (bx + u) * 32));
#pragma unroll
            for (uint32_t u = 0; u < kU; ++u) {
                const float4 b = *reinterpret_cast<const float4*>(ya + (bx + u) * 32);
                acc = fmaf(a[u].x, b.x, acc);
                acc = fmaf(a[u].y, b.y, acc);
                acc = fmaf(a[u].z, b.z, acc);
                acc = fmaf(a[u].w, b.w, acc);
            }
        }
        if (kU > 4 && bx + 4 <= nbox) {  // a half batch before the last slabs (D = 384: 8 + 4)
            float4 a[4];
#pragma unroll
            for (uint32_t u = 0; u < 4; ++u) a[u] = __ldg(reinterpret_cast<const float4*>(xa + (bx + u) * 32));
#pragma unroll
            for (uint32_t u = 0; u < 4; ++u) {
                const float4 b = *reinterpret_cast<const float4*>(ya + (bx + u) * 32);
                acc = fmaf(a[u].x, b.x, acc);
                acc = fmaf(a[u].y, b.y, acc);
                acc = fmaf(a[u].z, b.z, acc);
                acc = fmaf(a[u].w, b.w, acc);
            }
            bx += 4;
        }
        for (; bx < nbox; ++bx) {
            const float4 a = __ldg(reinterpret_cast<const float4*>(xa + bx * 32));
            const float4 b = *reinterpret_cast<const float4*>(ya + bx * 32);
            acc = fmaf(a.x, b.x, acc);
            acc = fmaf(a.y, b.y, acc);
            acc = fmaf(a.z, b.z, acc);
            acc = fmaf(a.w, b.w, acc);
        }
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    acc += __shfl_xor_sync(0xffffffffu, acc, 4);
    return acc;
}

// ------------------------------------------------------------------------------------------
// K4 (pass 1): exact FP32 rerank of the k′ candidates + top-k + certificate + T. One block per query.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024, 1)
    rerank_kernel(const float* __restrict__ base, uint32_t ds, const float* __restrict__ queries,
                  const uint64_t* __restrict__ cand_idx, const float* __restrict__ cand_bound,
                  const uint32_t* __restrict__ cand_cnt, uint32_t kp, uint32_t k, uint64_t* __restrict__ idx_out,
                  float* __restrict__ sim_out, uint32_t* __restrict__ cnt_out, uint32_t* __restrict__ cert_out,
                  float* __restrict__ kth_out, int certify, uint32_t* __restrict__ fb_ids,
                  uint32_t* __restrict__ fb_count, const uint32_t* __restrict__ row_map,
                  const unsigned long long* __restrict__ floor_keys) {
    extern __shared__ uint64_t keys[];  // p2(kp) keys, then the query (ds floats)
    const uint32_t q = blockIdx.x;
    const uint32_t ch = threadIdx.x & 7u, slot = threadIdx.x >> 3;  // 8 lanes per candidate
    const uint32_t nslots = blockDim.x >> 3;
    const uint32_t n = cand_cnt[q] < kp ? cand_cnt[q] : kp;
    uint32_t p2 = 1;
    while (p2 < kp) p2 <<= 1;
    const float* qv = queries + static_cast<size_t>(q) * ds;
    const uint32_t nbox = ds / 32;
    // the query in shared memory, so the registers hold eight of a row's slabs in flight
    float* q_s = reinterpret_cast<float*>(keys + p2);
    for (uint32_t d = threadIdx.x; d < ds; d += blockDim.x) q_s[d] = qv[d];
    __syncthreads();
    for (uint32_t j0 = 0; j0 < p2; j0 += nslots) {
        const uint32_t j = j0 + slot;
        const bool live = j < n;
        const uint64_t cand = live ? cand_idx[static_cast<size_t>(q) * kp + j] : 0;
        const uint32_t row = row_map && live ? row_map[cand] : static_cast<uint32_t>(cand);
        const float acc = dot_scan_order<8>(base + cand * ds, q_s, nbox, ch, live);
        if (ch == 0 && j < p2) keys[j] = live ? make_key(acc, row) : 0ull;
    }
    __syncthreads();
    block_bitonic_sort_desc(keys, p2);
    const uint32_t kk = n < k ? n : k;
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
        idx_out[static_cast<size_t>(q) * k + j] = j < kk ? key_row(keys[j]) : 0;
        sim_out[static_cast<size_t>(q) * k + j] = j < kk ? key_score(keys[j]) : 0.0f;
    }
    if (threadIdx.x == 0) {
        if (cnt_out) cnt_out[q] = kk;
        // Every row outside the k′ candidates has an exact score ≤ the k′-th upper bound; an exact
        // k-th score above it proves the top-k exact.
        // Rows outside the candidates: those the merge left out (bound ≤ the k′-th bound, when it
        // had k′) and those a full per-CTA list left out (bound ≤ the floor). With neither, every
        // row was a candidate and the result is exact as it stands.
        uint32_t ok = certify ? 1u : 0u;
        const unsigned long long fk = floor_keys ? floor_keys[q] : 0ull;
        if (certify && kk > 0 && (n >= kp || fk)) {
            float bound = n >= kp ? cand_bound[static_cast<size_t>(q) * kp + kp - 1] : -INFINITY;
            if (fk) bound = fmaxf(bound, key_score(fk));
            ok = key_score(keys[kk - 1]) > bound ? 1u : 0u;
        }
        cert_out[q] = ok;
        if (fb_count && !ok) fb_ids[atomicAdd(fb_count, 1u)] = q;  // for the FP32 scan
        // T: the exact k-th score among the candidates, a lower bound of the true k-th; with fewer
        // than k candidates (a sampled pass 1 over few rows) there is no bound.
        kth_out[q] = kk == k ? key_score(keys[kk - 1]) : -INFINITY;
    }
}

// ------------------------------------------------------------------------------------------
// Pass-2 helpers: gather the uncertified queries into a compact block, then rerank their
// threshold-collected rows exactly and write the top-k into their own output slots.
// ------------------------------------------------------------------------------------------
__global__ void gather_queries_kernel(const uint32_t* __restrict__ ids, uint32_t m, const uint8_t* __restrict__ q_lp,
                                      uint32_t row_bytes, uint8_t* __restrict__ q2_lp, const float* __restrict__ resid,
                                      float* __restrict__ resid2, const float* __restrict__ scale,
                                      float* __restrict__ scale2, const float* __restrict__ kth,
                                      float* __restrict__ thr2, const uint32_t* __restrict__ live) {
    const uint32_t i = blockIdx.x;
    if (live) {  // the count is on the device: rows past its 128-query block are not used
        m = *live;
        if (i >= (m + 127) / 128 * 128) return;
    }
    uint4* b = reinterpret_cast<uint4*>(q2_lp + static_cast<size_t>(i) * row_bytes);
    if (i >= m) {  // padding rows of the last 128-query block: zeros, not stale memory
        for (uint32_t t = threadIdx.x; t < row_bytes / 16; t += blockDim.x) b[t] = make_uint4(0, 0, 0, 0);
        return;
    }
    const uint32_t src = ids[i];
    const uint4* a = reinterpret_cast<const uint4*>(q_lp + static_cast<size_t>(src) * row_bytes);
    for (uint32_t t = threadIdx.x; t < row_bytes / 16; t += blockDim.x) b[t] = a[t];
    if (threadIdx.x == 0) {
        resid2[i] = resid[src];
        if (scale) scale2[i] = scale[src];
        thr2[i] = kth[src];
    }
}

// Pass 2's exact rerank runs as work items of up to kRerankChunk collected rows, so that a query
// with thousands of collected rows is spread over many blocks instead of one.
constexpr uint32_t kRerankChunk = 512;

// Keeps the best kk of keys[0, m) (distinct) in keys[0, kk), in no particular order.
NNDEX_DEVICE_INLINE void block_keep_best(uint64_t* keys, uint32_t m, uint32_t kk, BlockSelectScratch& sel) {
    const uint64_t kth = block_radix_kth(keys, m, kk, sel);
    if (threadIdx.x == 0) sel.count = 0;
    __syncthreads();
    for (uint32_t j0 = 0; j0 < m; j0 += blockDim.x) {
        const uint32_t j = j0 + threadIdx.x;
        const uint64_t key = j < m ? keys[j] : 0ull;
        __syncthreads();
        const bool take = j < m && key >= kth;
        const uint32_t pos = warp_append(&sel.count, take);
        if (take) keys[pos] = key;  // pos ≤ j: never overwrites a key not yet read
        __syncthreads();
    }
}

// Work item (i, c): rows [c·kRerankChunk, (c + 1)·kRerankChunk) of the collection of uncertified
// query i (ids[i]), re-scored exactly in the FP32 scan's order. Only rows whose exact score reaches T
// (the exact k-th score of pass 1, a lower bound of the true k-th) can be in the top-k, and the k
// rows that gave T are among the collected ones, so only those are kept; the item's best k of them
// go to its slot. `vecs` holds the vectors: the base by row, or (IVF) the list-ordered copy by
// collected position. Items past a query's collection (or of an overflowed one) return at once.
__global__ void __launch_bounds__(256)
    rerank_chunk_kernel(const float* __restrict__ vecs, uint32_t ds, const float* __restrict__ queries,
                        const uint32_t* __restrict__ ids, const uint32_t* __restrict__ rows2,
                        const uint32_t* __restrict__ cnt2, uint32_t cap2, uint32_t k, int by_query,
                        const uint32_t* __restrict__ live, const uint32_t* __restrict__ row_map,
                        const float* __restrict__ thr, uint64_t* __restrict__ slot_keys) {
    __shared__ uint64_t keys[kRerankChunk];
    __shared__ BlockSelectScratch sel;
    __shared__ uint32_t fill;
    const uint32_t i = blockIdx.x, c = blockIdx.y;
    if (live && i >= *live) return;
    const uint32_t q = ids[i];
    const uint32_t qrow = by_query ? q : i;  // collected rows and T indexed by query, or by position in ids
    const uint32_t total = cnt2[qrow];
    const uint32_t j_begin = c * kRerankChunk;
    if (total > cap2 || j_begin >= total) return;
    const uint32_t j_end = (total - j_begin) < kRerankChunk ? total : j_begin + kRerankChunk;
    const float t = thr[qrow];
    const uint32_t ch = threadIdx.x & 7u, slot = threadIdx.x >> 3, nslots = blockDim.x >> 3;
    const float* qv = queries + static_cast<size_t>(q) * ds;
    const uint32_t nbox = ds / 32;
    // the query in shared memory, so the registers hold eight of a row's slabs in flight
    extern __shared__ __align__(16) float q_s[];
    for (uint32_t d = threadIdx.x; d < ds; d += blockDim.x) q_s[d] = qv[d];
    if (threadIdx.x == 0) fill = 0;
    __syncthreads();
    for (uint32_t j0 = j_begin; j0 < j_end; j0 += nslots) {
        const uint32_t j = j0 + slot;
        const bool on = j < j_end;
        const uint32_t pos = on ? rows2[static_cast<size_t>(qrow) * cap2 + j] : 0u;
        const uint32_t row = row_map && on ? row_map[pos] : pos;
        const float acc = dot_scan_order<8>(vecs + static_cast<size_t>(row_map ? pos : row) * ds, q_s, nbox, ch, on);
        const bool take = ch == 0 && on && acc >= t;
        const uint32_t at = warp_append(&fill, take);
        if (take) keys[at] = make_key(acc, row);
    }
    __syncthreads();
    const uint32_t m = fill;
    const uint32_t kk = m < k ? m : k;
    if (m > kk) block_keep_best(keys, m, kk, sel);
    uint64_t* out = slot_keys + (static_cast<size_t>(i) * gridDim.y + c) * k;
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) out[j] = j < kk ? keys[j] : 0ull;
}

// Per uncertified query i: the best k over its items' slots, sorted, into the query's outputs (a
// collection that overflowed its buffer marks the query for the FP32 scan instead).
__global__ void __launch_bounds__(256)
    rerank_merge_kernel(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ cnt2, uint32_t cap2,
                        uint32_t k, int by_query, const uint32_t* __restrict__ live,
                        const uint64_t* __restrict__ slot_keys, uint32_t chunks, uint64_t* __restrict__ idx_out,
                        float* __restrict__ sim_out, uint32_t* __restrict__ cnt_out, uint32_t* __restrict__ ok_out) {
    extern __shared__ uint64_t keys[];  // chunks·k keys, at least p2(k)
    __shared__ BlockSelectScratch sel;
    const uint32_t i = blockIdx.x;
    if (live && i >= *live) return;
    const uint32_t q = ids[i];
    const uint32_t total = cnt2[by_query ? q : i];
    if (total > cap2) {  // the collected set overflowed: this query goes to the FP32 scan
        if (threadIdx.x == 0) ok_out[i] = 0;
        return;
    }
    const uint32_t items = (total + kRerankChunk - 1) / kRerankChunk;
    const uint64_t* src = slot_keys + static_cast<size_t>(i) * chunks * k;
    if (threadIdx.x == 0) sel.count = 0;
    __syncthreads();
    for (uint32_t j0 = 0; j0 < items * k; j0 += blockDim.x) {
        const uint32_t j = j0 + threadIdx.x;
        const uint64_t key = j < items * k ? src[j] : 0ull;
        const uint32_t at = warp_append(&sel.count, key != 0ull);
        if (key != 0ull) keys[at] = key;
    }
    __syncthreads();
    const uint32_t m = sel.count;
    __syncthreads();
    const uint32_t kk = m < k ? m : k;
    if (m > kk) block_keep_best(keys, m, kk, sel);
    uint32_t p2 = 1;
    while (p2 < kk) p2 <<= 1;
    for (uint32_t j = kk + threadIdx.x; j < p2; j += blockDim.x) keys[j] = 0ull;
    __syncthreads();
    block_bitonic_sort_desc(keys, p2);
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
        idx_out[static_cast<size_t>(q) * k + j] = j < kk ? key_row(keys[j]) : 0;
        sim_out[static_cast<size_t>(q) * k + j] = j < kk ? key_score(keys[j]) : 0.0f;
    }
    if (threadIdx.x == 0) {
        if (cnt_out) cnt_out[q] = kk;
        ok_out[i] = 1;
    }
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
template <bool kFp8, int kST, int kMode, bool kStreamA, bool kItems = false, int kQB = 1, bool kPair = false>
static cudaError_t launch_tc_impl(const TcArgs& a, cudaStream_t stream) {
    auto kern = scan_tc_kernel<kFp8, kST, kMode, kStreamA, kItems, kQB, kPair>;
    const uint32_t kp = kMode == 0 ? a.p.kprime : 0;
    if (kMode == 0 && (a.p.heap_k == 0 || a.p.heap_k > kp)) return cudaErrorInvalidValue;
    const size_t smem = tc_smem_bytes(a.p.nchunks, kp, kST, kFp8, kStreamA, kPair ? 3 : kQB);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    dim3 grid = kItems ? dim3(a.items, 1)
                       : (a.p.live_q ? dim3(a.live_items, 1) : dim3((a.p.nq + kM * kQB - 1) / (kM * kQB), a.nranges));
    if (kPair) {
        // two CTAs per (pair of query blocks, row range): live_items bounds the pairs
        grid.x = a.p.live_q ? 2u * a.live_items : (grid.x + 1u) / 2u * 2u;
    }
    // item mode: one CTA per item of the bound; each takes up to kItemsPerCta items from the counter
    // and exits, so CTAs of other streams' kernels get SMs between them
    TcParams p = a.p;
    p.kprime = kp;
    if (sync_check_enabled())
        set_launch_note("scan_tc fp8 %d stages %d mode %d stream_a %d items %d query blocks %d: grid (%u, %u), nq %u, "
                        "k' %u, tile stride %u, range rows %llu, rows %llu, smem %zu",
                        kFp8, kST, kMode, kStreamA, kItems, kQB, grid.x, grid.y, p.nq, kp, p.tile_stride,
                        (unsigned long long)p.range_rows, (unsigned long long)p.rows, smem);
    if (kPair) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = grid;
        cfg.blockDim = dim3(tc_threads<kMode>());
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaLaunchKernelEx(&cfg, kern, *a.tmap_q, *a.tmap_b, p);
        count_launch();
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    kern<<<grid, tc_threads<kMode>(), smem, stream>>>(*a.tmap_q, *a.tmap_b, p);
    count_launch();
    return cudaGetLastError();
}

template <bool kFp8, int kMode, bool kStreamA>
static cudaError_t launch_tc_stages(const TcArgs& a, cudaStream_t stream) {
    switch (a.stages) {
        case 4: return launch_tc_impl<kFp8, 4, kMode, kStreamA>(a, stream);
        case 3: return launch_tc_impl<kFp8, 3, kMode, kStreamA>(a, stream);
        case 2: return launch_tc_impl<kFp8, 2, kMode, kStreamA>(a, stream);
        default: return cudaErrorInvalidValue;
    }
}

// IVF item mode (BF16 only).
template <int kMode, bool kStreamA>
static cudaError_t launch_tc_items(const TcArgs& a, cudaStream_t stream) {
    switch (a.stages) {
        case 4: return launch_tc_impl<false, 4, kMode, kStreamA, true>(a, stream);
        case 3: return launch_tc_impl<false, 3, kMode, kStreamA, true>(a, stream);
        case 2: return launch_tc_impl<false, 2, kMode, kStreamA, true>(a, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_scan_tc(const TcArgs& a, bool fp8, int mode, cudaStream_t stream) {
    if (a.items) {
        if (fp8 || a.items > 0x7FFFFFFFu) return cudaErrorInvalidValue;
        if (mode == 0) return a.stream_a ? launch_tc_items<0, true>(a, stream) : launch_tc_items<0, false>(a, stream);
        return a.stream_a ? launch_tc_items<1, true>(a, stream) : launch_tc_items<1, false>(a, stream);
    }
    if (mode == 1 && a.qb == 2) {
        if (a.stream_a || a.p.range_rows % kN) return cudaErrorInvalidValue;
        switch (a.stages) {
            case 5: return fp8 ? launch_tc_impl<true, 5, 1, false, false, 2>(a, stream)
                               : launch_tc_impl<false, 5, 1, false, false, 2>(a, stream);
            case 4: return fp8 ? launch_tc_impl<true, 4, 1, false, false, 2>(a, stream)
                               : launch_tc_impl<false, 4, 1, false, false, 2>(a, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    if (mode == 1 && a.qb == 3) {
        if (a.stream_a || a.p.range_rows % kN) return cudaErrorInvalidValue;
        switch (a.stages) {
            case 8: return fp8 ? launch_tc_impl<true, 8, 1, false, false, 1, true>(a, stream)
                               : launch_tc_impl<false, 8, 1, false, false, 1, true>(a, stream);
            case 6: return fp8 ? launch_tc_impl<true, 6, 1, false, false, 1, true>(a, stream)
                               : launch_tc_impl<false, 6, 1, false, false, 1, true>(a, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    if (a.qb != 1) return cudaErrorInvalidValue;
    if (mode == 0) {
        if (a.stream_a) return fp8 ? launch_tc_stages<true, 0, true>(a, stream) : launch_tc_stages<false, 0, true>(a, stream);
        return fp8 ? launch_tc_stages<true, 0, false>(a, stream) : launch_tc_stages<false, 0, false>(a, stream);
    }
    if (a.stream_a) return fp8 ? launch_tc_stages<true, 1, true>(a, stream) : launch_tc_stages<false, 1, true>(a, stream);
    return fp8 ? launch_tc_stages<true, 1, false>(a, stream) : launch_tc_stages<false, 1, false>(a, stream);
}

cudaError_t launch_rerank(const RerankArgs& a, cudaStream_t stream) {
    uint32_t p2 = 1;
    while (p2 < a.kp) p2 <<= 1;
    // One block per query; a small batch leaves most SMs idle, so its blocks take 1024 threads (128
    // candidates re-scored at once instead of 32) to keep more row loads in flight.
    const uint32_t threads = a.nq < 64 ? 1024u : 256u;
    const size_t smem = p2 * sizeof(uint64_t) + static_cast<size_t>(a.ds) * sizeof(float);
    if (smem > 48 * 1024) {
        const cudaError_t ea =
            cudaFuncSetAttribute(rerank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (ea != cudaSuccess) return ea;
    }
    rerank_kernel<<<a.nq, threads, smem, stream>>>(a.base, a.ds, a.queries, a.cand_idx, a.cand_sim,
                                                               a.cand_cnt, a.kp, a.k, a.idx_out, a.sim_out,
                                                               a.cnt_out, a.cert_out, a.kth_out, a.certify ? 1 : 0,
                                                               a.fb_ids, a.fb_count, a.row_map, a.floor_keys);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_gather_queries(const uint32_t* ids, uint32_t m, const void* q_lp, uint32_t row_bytes, void* q2_lp,
                                  const float* resid, float* resid2, const float* scale, float* scale2,
                                  const float* kth, float* thr2, cudaStream_t stream, const uint32_t* live) {
    if (m == 0) return cudaSuccess;
    // One block per row of the padded query buffer (m rounded up to the 128-query block; with a
    // device count `live`, m is its bound).
    const uint32_t m_alloc = (m + 127) / 128 * 128;
    gather_queries_kernel<<<m_alloc, 128, 0, stream>>>(ids, m, static_cast<const uint8_t*>(q_lp), row_bytes,
                                                 static_cast<uint8_t*>(q2_lp), resid, resid2, scale, scale2, kth, thr2,
                                                 live);
    count_launch();
    return cudaGetLastError();
}

uint32_t rerank_chunks(uint32_t cap2) { return (cap2 + kRerankChunk - 1) / kRerankChunk; }

cudaError_t launch_rerank_collected(const float* vecs, uint32_t ds, const float* queries, const uint32_t* ids,
                                    uint32_t m, const uint32_t* rows2, const uint32_t* cnt2, uint32_t cap2, uint32_t k,
                                    const float* thr, uint64_t* slot_keys, uint64_t* idx_out, float* sim_out,
                                    uint32_t* cnt_out, uint32_t* ok_out, cudaStream_t stream, bool by_query,
                                    const uint32_t* live, const uint32_t* row_map) {
    if (m == 0) return cudaSuccess;
    const uint32_t chunks = rerank_chunks(cap2);
    if (k == 0 || k > kRerankChunk || chunks > 65535u) return cudaErrorInvalidValue;
    const size_t qsmem = static_cast<size_t>(ds) * sizeof(float);
    if (qsmem > 48 * 1024) {
        const cudaError_t ea = cudaFuncSetAttribute(rerank_chunk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    static_cast<int>(qsmem));
        if (ea != cudaSuccess) return ea;
    }
    rerank_chunk_kernel<<<dim3(m, chunks), 256, qsmem, stream>>>(vecs, ds, queries, ids, rows2, cnt2, cap2, k,
                                                                by_query ? 1 : 0, live, row_map, thr, slot_keys);
    uint32_t p2 = 1;
    while (p2 < k) p2 <<= 1;
    const size_t smem = std::max<size_t>(static_cast<size_t>(chunks) * k, p2) * sizeof(uint64_t);
    auto kern = rerank_merge_kernel;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    kern<<<m, 256, smem, stream>>>(ids, cnt2, cap2, k, by_query ? 1 : 0, live, slot_keys, chunks, idx_out, sim_out,
                                   cnt_out, ok_out);
    count_launch(2);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// Device-side fallback of a certificate: the queries whose certificate failed are compacted,
// gathered, re-run on the FP32 scan (whose launch returns at once when there are none) and their
// results scattered back, all on the stream, with no host round trip.
// ------------------------------------------------------------------------------------------

// One block of 1024 threads: ids[0..m) = the indices i < n with flags[i] == 0, in order; count[0] = m.
// With `live`, only the first live[0] flags count.
__global__ void __launch_bounds__(1024) compact_zero_flags_kernel(const uint32_t* __restrict__ flags, uint32_t n,
                                                                  uint32_t* __restrict__ ids,
                                                                  uint32_t* __restrict__ count,
                                                                  const uint32_t* __restrict__ live) {
    __shared__ uint32_t warp_sum[32];
    __shared__ uint32_t base;
    if (live && *live < n) n = *live;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t i0 = 0; i0 < n; i0 += 1024) {
        const uint32_t i = i0 + threadIdx.x;
        const bool take = i < n && flags[i] == 0;
        const uint32_t ballot = __ballot_sync(0xFFFFFFFFu, take);
        if (lane == 0) warp_sum[warp] = __popc(ballot);
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t w = 0; w < 32; ++w) {
            const uint32_t v = warp_sum[w];
            before += w < warp ? v : 0u;
            total += v;
        }
        if (take) ids[base + before + __popc(ballot & ((1u << lane) - 1u))] = i;
        __syncthreads();
        if (threadIdx.x == 0) base += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) count[0] = base;
}

// Row i of dst (stride ds floats) = row ids[i] of src for i < count[0], zeros for the rest of n.
__global__ void gather_rows_kernel(const float* __restrict__ src, uint32_t ds, const uint32_t* __restrict__ ids,
                                   const uint32_t* __restrict__ count, float* __restrict__ dst) {
    const uint32_t i = blockIdx.x;
    float4* d = reinterpret_cast<float4*>(dst + static_cast<size_t>(i) * ds);
    if (i >= count[0]) {
        for (uint32_t t = threadIdx.x; t < ds / 4; t += blockDim.x) d[t] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float4* a = reinterpret_cast<const float4*>(src + static_cast<size_t>(ids[i]) * ds);
    for (uint32_t t = threadIdx.x; t < ds / 4; t += blockDim.x) d[t] = a[t];
}

// The results of re-run query i (< count[0]) into the slots of query ids[i].
__global__ void scatter_results_kernel(const uint64_t* __restrict__ fb_idx, const float* __restrict__ fb_sim,
                                       const uint32_t* __restrict__ fb_cnt, const uint32_t* __restrict__ ids,
                                       const uint32_t* __restrict__ count, uint32_t k, uint64_t* __restrict__ idx,
                                       float* __restrict__ sim, uint32_t* __restrict__ cnt) {
    const uint32_t i = blockIdx.x;
    if (i >= count[0]) return;
    const uint32_t q = ids[i];
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
        idx[static_cast<size_t>(q) * k + j] = fb_idx[static_cast<size_t>(i) * k + j];
        sim[static_cast<size_t>(q) * k + j] = fb_sim[static_cast<size_t>(i) * k + j];
    }
    if (threadIdx.x == 0 && cnt) cnt[q] = fb_cnt[i];
}

void launch_compact_zero_flags(const uint32_t* flags, uint32_t n, uint32_t* ids, uint32_t* count, cudaStream_t s,
                               const uint32_t* live) {
    compact_zero_flags_kernel<<<1, 1024, 0, s>>>(flags, n, ids, count, live);
    count_launch();
}

void launch_gather_rows(const float* src, uint32_t ds, const uint32_t* ids, const uint32_t* count, uint32_t n,
                        float* dst, cudaStream_t s) {
    if (n == 0) return;
    gather_rows_kernel<<<n, 128, 0, s>>>(src, ds, ids, count, dst);
    count_launch();
}

void launch_scatter_results(const uint64_t* fb_idx, const float* fb_sim, const uint32_t* fb_cnt, const uint32_t* ids,
                            const uint32_t* count, uint32_t n, uint32_t k, uint64_t* idx, float* sim, uint32_t* cnt,
                            cudaStream_t s) {
    if (n == 0) return;
    scatter_results_kernel<<<n, 128, 0, s>>>(fb_idx, fb_sim, fb_cnt, ids, count, k, idx, sim, cnt);
    count_launch();
}

// FP8: per 256-row tile of the base, {smallest, largest} scale over the tile's rows (rows past the
// base excluded; a tile without rows gets {+inf, 0}). One warp per tile.
__global__ void tile_scale_kernel(const float* __restrict__ row_scale, uint64_t rows, uint64_t tiles,
                                  float2* __restrict__ out) {
    const uint64_t t = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (t >= tiles) return;
    float lo = INFINITY, hi = 0.0f;
    for (uint32_t j = lane; j < 256; j += 32) {
        const uint64_t r = t * 256 + j;
        if (r < rows) {
            lo = fminf(lo, row_scale[r]);
            hi = fmaxf(hi, row_scale[r]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
    }
    if (lane == 0) out[t] = make_float2(lo, hi);
}

void launch_tile_scale(const float* row_scale, uint64_t rows, uint64_t tiles, float2* out, cudaStream_t s) {
    if (tiles == 0) return;
    tile_scale_kernel<<<static_cast<uint32_t>((tiles * 32 + 255) / 256), 256, 0, s>>>(row_scale, rows, tiles, out);
    count_launch();
}

// Largest row residual norm (the ε of the certificate), by a grid-stride max.
__global__ void max_reduce_kernel(const float* __restrict__ v, uint64_t n, unsigned int* __restrict__ out) {
    float m = 0.0f;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        m = fmaxf(m, v[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));  // non-negative floats order as uints
}

cudaError_t launch_max_reduce(const float* v, uint64_t n, unsigned int* out, cudaStream_t stream) {
    max_reduce_kernel<<<148 * 4, 256, 0, stream>>>(v, n, out);
    count_launch();
    return cudaGetLastError();
}

}  // namespace nndex
