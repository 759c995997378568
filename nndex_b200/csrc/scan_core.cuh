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

// When a query's buffer could overflow on the next tile (or, after the last tile, holds more than
// k), one warp radix-selects its exact k best, compacts, and raises its threshold. Called by every
// consumer thread after insert(); ends synchronised when it did any work.
template <int QB, int NCW>
NNDEX_DEVICE_INLINE void scan_flush(bool last, uint32_t nqg, uint32_t k, uint32_t cap, uint32_t warp, uint32_t lane,
                                    uint32_t* cnt, uint64_t* thr, uint64_t* cand, uint32_t* hist) {
    using S = ScanShape<QB, NCW>;
    bool need = false;
#pragma unroll
    for (int b = 0; b < QB; ++b)
        if (static_cast<uint32_t>(b) < nqg) need |= last ? (cnt[b] > k) : (cnt[b] + S::kTileRows > cap);
    if (!need) return;
    for (uint32_t b = warp; b < nqg; b += S::kConsumers) {
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
    named_bar_sync(1, S::kConsumers * 32);
}

}  // namespace nndex
