// scan_core.cuh — the consumer side of the FP32 scan, shared by the exact scan (K2, scan_fp32.cu)
// and the IVF list scan (K9, ivf_search.cu).
//
// A tile is NCW·32 rows; each 128-byte slab of it (32 floats of every row, 128-byte swizzle) arrives
// in a ring stage filled by one producer warp. Consumer warp w = qg·(2·NCW) + half·NCW + rgrp owns
// tile rows [32·rgrp, 32·rgrp + 32), the 16-byte chunks 4·half + dg of every slab, and the QW
// queries qg·QW … qg·QW + QW − 1 of the CTA's QB (QB = 16 runs two query groups: twice the warps,
// half the registers each, for latency hiding). Lane (rg = lane / 4, dg = lane % 4) keeps rows
// rg + 8i (i < 4) × QW queries of FP32 partial sums. With the 128-byte swizzle
// (chunk' = chunk ^ (row % 8) = chunk ^ rg) every row load is conflict-free and every query load
// is a 4-address broadcast.
//
// The FMA order of one (row, query) pair is fixed: per chunk position, the slab's 4 products in
// order, slab after slab; the 4 positions of a half combine as (p0 + p1) + (p2 + p3) by two xor
// shuffles; the halves add as half0 + half1 through shared memory. It depends on nothing else
// (batch, tile, grid), so every path that scores a row in this order gets the same bits; the
// rerank's dot_scan_order (scan_tc.cu) restates it.
#pragma once

#include "common.cuh"
#include "select.cuh"

namespace nndex {

template <int QB, int NCW>
struct ScanShape {
    static constexpr int kQW = QB < 8 ? QB : 8;            // queries per consumer warp
    static constexpr int kQG = QB / kQW;                     // query groups per CTA (1 or 2)
    static constexpr int kConsumers = 2 * NCW * kQG;         // consumer warps
    static constexpr int kThreads = (kConsumers + 1) * 32;   // + the producer warp
    static constexpr int kTileRows = NCW * 32;
    static constexpr uint32_t kStageBytes = kTileRows * 128;
    static constexpr int kXchg = 4 * (kQW < 4 ? 1 : kQW / 4);  // values a lane hands its partner per tile
};

// Host-side mirror of ScanShape's shared-memory terms (qb = queries per CTA).
__host__ __device__ constexpr uint32_t scan_consumers(uint32_t qb, uint32_t ncw) {
    return 2 * ncw * (qb <= 8 ? 1 : qb / 8);
}
__host__ __device__ constexpr uint32_t scan_xchg_per_lane(uint32_t qb) {
    return 4 * ((qb < 8 ? qb : 8) < 4 ? 1 : (qb < 8 ? qb : 8) / 4);
}

template <int QB, int NCW, int ST>
struct ScanConsumer {
    using S = ScanShape<QB, NCW>;
    static constexpr int QW = S::kQW;
    static_assert((ST & (ST - 1)) == 0, "ring depth must be a power of two");

    uint32_t lane, qg, half, rgrp, dg, rg;
    uint32_t x_base, q_base, q_stride;
    float* my_x;
    const float* peer_x;

    NNDEX_DEVICE_INLINE ScanConsumer(uint32_t warp, uint32_t lane_, const uint8_t* stage_base, const float* q_s,
                                     uint32_t dq, float* xchg)
        : lane(lane_) {
        qg = warp / (2 * NCW);
        half = (warp / NCW) & 1u;
        rgrp = warp % NCW;
        dg = lane & 3u;
        rg = lane >> 2;
        const uint32_t ch = dg + 4 * half;
        x_base = smem_u32(stage_base) + (rgrp * 32 + rg) * 128 + ((ch ^ rg) * 16);
        q_stride = dq * 4;
        q_base = smem_u32(q_s) + ch * 16 + qg * QW * q_stride;
        const uint32_t peer = qg * (2 * NCW) + (1 - half) * NCW + rgrp;
        my_x = xchg + (warp * 32 + lane) * S::kXchg;
        peer_x = xchg + (peer * 32 + lane) * S::kXchg;
    }

    // One tile: nbox slabs from the ring (starting at ring position `it`, advanced), each released
    // to the producer once its values are consumed.
    NNDEX_DEVICE_INLINE void accumulate(float (&acc)[4][QW], uint32_t nbox, uint32_t& it, uint64_t* full_bar,
                                        uint64_t* empty_bar, volatile uint32_t* abort_flag, uint32_t* status) const {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int b = 0; b < QW; ++b) acc[i][b] = 0.0f;
#pragma unroll 1
        for (uint32_t bx = 0; bx < nbox; ++bx, ++it) {
            const uint32_t s = it & (ST - 1), parity = (it / ST) & 1u;
            // Queries do not depend on the slab: load them before waiting for it.
            float4 qv[QW];
#pragma unroll
            for (int b = 0; b < QW; ++b) qv[b] = lds128(q_base + b * q_stride + bx * 128);
            if (!*abort_flag && !mbar_wait_bounded(&full_bar[s], parity, kWaitBudgetCycles)) {
                *abort_flag = 1;
                record_status(status, kStatusTimeout);
            }
            const uint32_t xa = x_base + s * S::kStageBytes;
            float4 x[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) x[i] = lds128(xa + i * 8 * 128);
            // 4·QW independent accumulators per component: no FMA dependency stalls.
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int b = 0; b < QW; ++b) acc[i][b] = fmaf(x[i].x, qv[b].x, acc[i][b]);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int b = 0; b < QW; ++b) acc[i][b] = fmaf(x[i].y, qv[b].y, acc[i][b]);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int b = 0; b < QW; ++b) acc[i][b] = fmaf(x[i].z, qv[b].z, acc[i][b]);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int b = 0; b < QW; ++b) acc[i][b] = fmaf(x[i].w, qv[b].w, acc[i][b]);
            // The slab's values are consumed (the FMAs above read them): release it to the producer.
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty_bar[s]);
        }
    }

    // Completes the tile's scores (xor shuffles, then the partner half through shared memory) and
    // appends every key that beats its query's running k-th key. row_key(r) maps a tile row to the
    // row index the key carries. Ends with the consumers synchronised.
    template <class RowKey>
    NNDEX_DEVICE_INLINE void insert(float (&acc)[4][QW], uint64_t tile_row0, uint64_t row_end, uint32_t nqg,
                                    RowKey row_key, const uint64_t* thr, uint32_t* cnt, uint64_t* cand, uint32_t cap,
                                    uint32_t* status) const {
        constexpr uint32_t nthreads_c = S::kConsumers * 32;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int b = 0; b < QW; ++b) {
                float v = acc[i][b];
                v += __shfl_xor_sync(0xffffffffu, v, 1);
                v += __shfl_xor_sync(0xffffffffu, v, 2);
                acc[i][b] = v;
            }
        // Lane dg publishes its sums of the queries b ≡ dg (mod 4). Half 0 inserts rows i = 0, 1 and
        // half 1 rows i = 2, 3; both add (half0 + half1).
        {
            int j = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int b = 0; b < QW; ++b)
                    if ((b & 3) == static_cast<int>(dg)) {
                        my_x[j] = acc[i][b];
                        ++j;
                    }
        }
        named_bar_sync(1, nthreads_c);
        const uint64_t r0 = tile_row0 + rgrp * 32 + rg;
        {
            int j = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int b = 0; b < QW; ++b)
                    if ((b & 3) == static_cast<int>(dg)) {
                        const float other = peer_x[j];
                        ++j;
                        const uint32_t bq = qg * QW + b;
                        if ((i >> 1) == static_cast<int>(half) && bq < nqg) {
                            const uint64_t r = r0 + 8 * i;
                            if (r < row_end) {
                                const float v = half == 0 ? acc[i][b] + other : other + acc[i][b];
                                const uint64_t key = make_key(v, row_key(r));
                                if (key > thr[bq]) {
                                    const uint32_t pos = atomicAdd(&cnt[bq], 1u);
                                    if (pos < cap)
                                        cand[static_cast<size_t>(bq) * cap + pos] = key;
                                    else
                                        record_status(status, kStatusOverflow);
                                }
                            }
                        }
                    }
        }
        named_bar_sync(1, nthreads_c);
    }
};

// The wide consumer (K2 at 8 or 16 queries per CTA): each of the W consumer warps owns 16 tile rows
// and ALL of the CTA's QB queries, so every row value is read from shared memory once. Lane
// (rg = lane / 8, dg = lane % 8) keeps rows 16w + rg + 4i (i < 4) × QB queries of partial sums for
// chunk position dg (16 bytes) of every slab: a row load is one 128-byte row per 8 lanes
// (conflict-free under the 128-byte swizzle) and a query load is 8 consecutive chunks, one full
// wavefront broadcast to the 4 row groups. The next slab's rows are loaded before the current one
// is multiplied, and the queries are loaded four at a time between their FMAs, so shared-memory
// traffic is spread over the FMA stream instead of bursting after each barrier.
//
// The FMA order per (row, query) is ScanConsumer's: per chunk position the slab's 4 products in
// order, slab after slab, then ((p0 + p1) + (p2 + p3)) + ((p4 + p5) + (p6 + p7)) over the 8
// positions. The tile's scores are completed by a reduce-scatter butterfly over the 8 lanes of a
// row group (xor 1, 2, 4, halving the values a lane keeps at each step): the same addition tree,
// and IEEE addition commutes, so every score has ScanConsumer's bits. Each lane ends with one row
// × QB/2 queries and inserts those; no shared-memory exchange is needed.
// A position in a ring of ST stages: the stage and the parity of its current phase.
template <int ST>
struct RingPos {
    uint32_t s = 0, phase = 0;
    NNDEX_DEVICE_INLINE RingPos next() const {
        RingPos n = *this;
        if (++n.s == ST) {
            n.s = 0;
            n.phase ^= 1u;
        }
        return n;
    }
};

template <int QB, int W, int ST>
struct ScanConsumerWide {
    static_assert(QB == 1 || QB == 2 || QB == 4 || QB == 8 || QB == 16, "the wide consumer takes 1-16 queries");
    static constexpr int kGQ = QB < 4 ? QB : 4;  // queries per FMA group
    static constexpr int kTileRows = 16 * W;
    static constexpr uint32_t kStageBytes = kTileRows * 128;
    static constexpr int kHalf = QB >= 2 ? QB / 2 : 1;  // values a lane inserts
    // Queries in shared memory slab-major: [dq / 32][QB][32] floats, so a slab's query chunks sit
    // at fixed offsets (b · 128 bytes) from the slab's base.
    static constexpr uint32_t kQSlabBytes = QB * 128;
    NNDEX_DEVICE_INLINE static uint32_t q_slab_index(uint32_t b, uint32_t d) { return ((d >> 5) * QB + b) * 32 + (d & 31u); }

    uint32_t lane, rg, dg, warp;
    uint32_t x_base0, x_base1;  // row chunk address (stage 0) for rows i = 0, 2 and i = 1, 3
    uint32_t q_base;            // shared address of this lane's chunk of query 0 in slab 0

    NNDEX_DEVICE_INLINE ScanConsumerWide(uint32_t warp_, uint32_t lane_, const uint8_t* stage_base, const float* q_s)
        : lane(lane_), warp(warp_) {
        rg = lane >> 3;
        dg = lane & 7u;
        // row 16w + rg + 4i: (row % 8) = rg + 4·(i % 2), the 128-byte swizzle's chunk xor
        const uint32_t row0 = warp * 16 + rg;
        x_base0 = smem_u32(stage_base) + row0 * 128 + ((dg ^ rg) * 16);
        x_base1 = smem_u32(stage_base) + (row0 + 4) * 128 + ((dg ^ (rg + 4)) * 16);
        q_base = smem_u32(q_s) + dg * 16;
    }

    NNDEX_DEVICE_INLINE void load_rows(float4 (&x)[4], RingPos<ST> r) const {
        const uint32_t off = r.s * kStageBytes;
        x[0] = lds128(x_base0 + off);
        x[1] = lds128(x_base1 + off);
        x[2] = lds128(x_base0 + off + 8 * 128);
        x[3] = lds128(x_base1 + off + 8 * 128);
    }

    NNDEX_DEVICE_INLINE void wait_full(uint64_t* full_bar, RingPos<ST> r, volatile uint32_t* abort_flag,
                                       uint32_t* status) const {
        if (mbar_try_wait(&full_bar[r.s], r.phase)) return;
        if (!*abort_flag && !mbar_wait_bounded(&full_bar[r.s], r.phase, kWaitBudgetCycles)) {
            *abort_flag = 1;
            record_status(status, kStatusTimeout);
        }
    }

    // acc += the products of rows x and queries [4·G0, 4·G1) at shared address q (chunk dg), in
    // component order. The queries are written once before the consumers start; explicit
    // shared-memory loads (the address space is not left for the compiler to infer). Four queries
    // at a time: 16 independent FMAs separate the dependent ones of an accumulator.
    template <int G0, int G1>
    NNDEX_DEVICE_INLINE static void fma_groups(float (&acc)[4][QB], const float4 (&x)[4], uint32_t q) {
#pragma unroll
        for (int b0 = kGQ * G0; b0 < kGQ * G1; b0 += kGQ) {
            float4 qv[kGQ];
#pragma unroll
            for (int j = 0; j < kGQ; ++j) qv[j] = lds128(q + (b0 + j) * 128);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < kGQ; ++j) acc[i][b0 + j] = fmaf(x[i].x, qv[j].x, acc[i][b0 + j]);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < kGQ; ++j) acc[i][b0 + j] = fmaf(x[i].y, qv[j].y, acc[i][b0 + j]);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < kGQ; ++j) acc[i][b0 + j] = fmaf(x[i].z, qv[j].z, acc[i][b0 + j]);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < kGQ; ++j) acc[i][b0 + j] = fmaf(x[i].w, qv[j].w, acc[i][b0 + j]);
        }
    }

    // Every lane arrives (the empty barriers count W·32 arrivals) once its FMAs have used the
    // slab's row values, i.e. once its loads of the stage have completed.
    NNDEX_DEVICE_INLINE void release(uint64_t* empty_bar, RingPos<ST> r) const { mbar_arrive(&empty_bar[r.s]); }

    // One slab with the rows in x (ring position it) while the next slab's rows go to xn: the
    // next stage's barrier is tested before the first query group's FMAs and the branch on it
    // (and the row loads it guards) comes after them, so neither the test nor the loads' latency
    // holds up the FMA stream.
    NNDEX_DEVICE_INLINE void slab(float (&acc)[4][QB], const float4 (&x)[4], float4 (&xn)[4], bool more,
                                  RingPos<ST> cur, uint32_t q, uint64_t* full_bar, uint64_t* empty_bar,
                                  volatile uint32_t* abort_flag, uint32_t* status) const {
        const RingPos<ST> nxt = cur.next();
        const bool ready = !more || mbar_try_wait(&full_bar[nxt.s], nxt.phase);
        fma_groups<0, 1>(acc, x, q);
        if (more) {
            if (!ready && !*abort_flag &&
                !mbar_wait_bounded_suspend(&full_bar[nxt.s], nxt.phase, kWaitBudgetCycles, 20000)) {
                *abort_flag = 1;
                record_status(status, kStatusTimeout);
            }
            load_rows(xn, nxt);
        }
        fma_groups<1, QB / kGQ>(acc, x, q);
        release(empty_bar, cur);
    }

    // One tile: nbox slabs from the ring (starting at ring position `pos`, advanced), each released
    // to the producer once its row values have been used (two register sets, alternating).
    NNDEX_DEVICE_INLINE void accumulate(float (&acc)[4][QB], uint32_t nbox, RingPos<ST>& pos, uint64_t* full_bar,
                                        uint64_t* empty_bar, volatile uint32_t* abort_flag, uint32_t* status) const {
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int b = 0; b < QB; ++b) acc[i][b] = 0.0f;
        float4 xa[4], xb[4];
        wait_full(full_bar, pos, abort_flag, status);
        load_rows(xa, pos);
        uint32_t q = q_base;
#pragma unroll 1
        for (uint32_t bx = 0; bx < nbox; bx += 2) {
            slab(acc, xa, xb, bx + 1 < nbox, pos, q, full_bar, empty_bar, abort_flag, status);
            pos = pos.next();
            q += kQSlabBytes;
            if (bx + 1 >= nbox) break;
            slab(acc, xb, xa, bx + 2 < nbox, pos, q, full_bar, empty_bar, abort_flag, status);
            pos = pos.next();
            q += kQSlabBytes;
        }
    }

    // One butterfly step over lanes xor m: a lane whose bit m is clear keeps the first half of its
    // values and receives the partner's share of them; the other lane keeps the second half.
    template <int N>
    NNDEX_DEVICE_INLINE static void halve(const float (&v)[N], float (&out)[N / 2], uint32_t m, bool upper) {
#pragma unroll
        for (int j = 0; j < N / 2; ++j) {
            const float send = upper ? v[j] : v[j + N / 2];
            const float keep = upper ? v[j + N / 2] : v[j];
            out[j] = keep + __shfl_xor_sync(0xffffffffu, send, m);
        }
    }

    // Completes the tile's scores and appends every key that beats its query's running k-th key.
    // row_key(r) maps a tile row to the row index the key carries. Ends with the consumers
    // synchronised.
    template <class RowKey>
    NNDEX_DEVICE_INLINE void insert(const float (&acc)[4][QB], uint64_t tile_row0, uint64_t row_end, uint32_t nqg,
                                    RowKey row_key, const uint64_t* thr, uint32_t* cnt, uint64_t* cand, uint32_t cap,
                                    uint32_t* status) const {
        float v4[4 * QB];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int b = 0; b < QB; ++b) v4[i * QB + b] = acc[i][b];
        float v2[2 * QB], v1[QB], v0[kHalf];
        halve<4 * QB>(v4, v2, 1, (dg & 1u) != 0);   // keeps rows {0,1} or {2,3}
        halve<2 * QB>(v2, v1, 2, (dg & 2u) != 0);   // keeps one row of those two
        bool inserts = true;
        if constexpr (QB >= 2) {
            halve<QB>(v1, v0, 4, (dg & 4u) != 0);   // keeps queries [0, QB/2) or [QB/2, QB)
        } else {
            // one value left: the last step adds the partner's (S0 + S1 in both lanes: addition
            // commutes) and the lane whose bit is clear inserts it
            v0[0] = v1[0] + __shfl_xor_sync(0xffffffffu, v1[0], 4);
            inserts = (dg & 4u) == 0;
        }
        const uint32_t i_l = 2 * (dg & 1u) + ((dg >> 1) & 1u);
        const uint64_t r = tile_row0 + warp * 16 + rg + 4 * i_l;
        const uint32_t b0 = QB >= 2 ? kHalf * (dg >> 2) : 0u;
        if (r < row_end && inserts) {
            const uint32_t rk = row_key(r);
#pragma unroll
            for (int t = 0; t < kHalf; ++t) {
                const uint32_t bq = b0 + t;
                if (bq < nqg) {
                    const uint64_t key = make_key(v0[t], rk);
                    if (key > thr[bq]) {
                        const uint32_t pos = atomicAdd(&cnt[bq], 1u);
                        if (pos < cap)
                            cand[static_cast<size_t>(bq) * cap + pos] = key;
                        else
                            record_status(status, kStatusOverflow);
                    }
                }
            }
        }
        named_bar_sync(1, W * 32);
    }
};

// When a query's buffer could overflow on the next tile (or, after the last tile, holds more than
// k), one warp radix-selects its exact k best, compacts, and raises its threshold. Called by every
// consumer thread after insert(); ends synchronised when it did any work.
template <int QB, int kConsumers, int kTileRows>
NNDEX_DEVICE_INLINE void scan_flush_g(bool last, uint32_t nqg, uint32_t k, uint32_t cap, uint32_t warp,
                                      uint32_t lane, uint32_t* cnt, uint64_t* thr, uint64_t* cand, uint32_t* hist) {
    bool need = false;
#pragma unroll
    for (int b = 0; b < QB; ++b)
        if (static_cast<uint32_t>(b) < nqg) need |= last ? (cnt[b] > k) : (cnt[b] + kTileRows > cap);
    if (!need) return;
    // Every consumer has read the counts (and so made the same decision) before any warp
    // rewrites them: a warp that read a count already compacted would skip the barrier below.
    named_bar_sync(1, kConsumers * 32);
    for (uint32_t b = warp; b < nqg; b += kConsumers) {
        const uint32_t n = cnt[b] < cap ? cnt[b] : cap;
        if (n > k) {
            uint64_t* buf = cand + static_cast<size_t>(b) * cap;
            const uint64_t kth = warp_radix_kth(buf, n, k, hist + warp * 256);
            const uint32_t m = warp_compact_ge(buf, n, kth);
            if (lane == 0) {
                cnt[b] = m;
                thr[b] = kth;
            }
        }
    }
    named_bar_sync(1, kConsumers * 32);
}

template <int QB, int NCW>
NNDEX_DEVICE_INLINE void scan_flush(bool last, uint32_t nqg, uint32_t k, uint32_t cap, uint32_t warp, uint32_t lane,
                                    uint32_t* cnt, uint64_t* thr, uint64_t* cand, uint32_t* hist) {
    using S = ScanShape<QB, NCW>;
    scan_flush_g<QB, S::kConsumers, S::kTileRows>(last, nqg, k, cap, warp, lane, cnt, thr, cand, hist);
}

}  // namespace nndex
