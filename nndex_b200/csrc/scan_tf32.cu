// scan_tf32.cu — K12: FP32-accurate candidate scan on the tensor cores for small query batches.
//
// Replaces the FP32 FMA stream of the exact scan (src/gpu.rs score pass, src/cpu.rs dot loop) where
// that stream, not HBM, bounds it: at 9–16 queries per batch the FP32 scan needs 2·B FLOPs per base
// byte and runs out of issue slots near 60 % of the HBM rate. Here the tensor cores do the
// products; the CUDA cores only split each staged base value in two:
//
//   x = xb + xs, xb = x with its 13 low mantissa bits cleared (exact in TF32), xs = x − xb (exact),
//   and likewise q = qb + qs for the queries (split once, before the launch).
//   s̃ = xb·qb + xb·qs + xs·qb   (three kind::tf32 MMAs per K step, FP32 accumulation in TMEM)
//
// |xs| < 2⁻¹⁰|x|, and the MMA reads xs and qs with 10 mantissa bits, so each product is off by less
// than 3·2⁻²⁰·|x_i q_i|: s̃ is FP32-accurate, not bit-identical to the FP32 scan's FMA chain. It
// therefore only ranks candidates. Each CTA keeps, per query, the k′ rows with the best upper
// bound u = s̃ + ε, where ε bounds |FP32 scan-order score − s̃|. The merge keeps each query's k′
// best, and the exact rerank (K4: the FP32 scan's own summation order) returns the top-k with the
// certificate "exact k-th > k′-th bound". So a certified query's rows and scores are bit for bit
// those of the FP32 scan. An uncertified query is re-run on the FP32 scan by the host.
//
// Layout: one CTA per (row range, block of 16 queries); tiles of 128 base rows × one 128-byte slab
// (32 FP32 values) per ring stage, loaded by TMA with the 128-byte swizzle. In each stage, after
// the split, xb sits in place of x, then xs, qb and qs. The MMA is M = 128 rows × N = 16 queries
// × K = 8, so the accumulator is 16 TMEM columns per tile (two tiles in flight: 32 columns). The
// epilogue thread of TMEM lane r owns base row r of the tile: it reads its 16 scores and appends
// each (u, row) key that beats its query's running k′-th key. Selection is the FP32 scan's own
// machinery (scan_flush_g).
//
// Warps: 0 TMA producer, 1 MMA issuer, 2–5 split, 6–9 epilogue. Every wait is bounded; on a
// timeout the kernel records it in the status word, stops issuing, drains its copies and the
// tensor core's barrier arrivals, frees its TMEM and exits.
#include <cuda.h>

#include <algorithm>

#include "common.cuh"
#include "internal.h"
#include "scan_core.cuh"
#include "select.cuh"
#include "tc.cuh"

namespace nndex {

namespace {
constexpr int kTfM = 128;                             // base rows per tile (MMA M, TMEM lanes)
constexpr int kTfN = 16;                              // queries per CTA (MMA N)
constexpr uint32_t kTfX = kTfM * 128;                 // one slab of the tile: 16 KB
constexpr uint32_t kTfQ = kTfN * 128;                 // one slab of the queries: 2 KB
constexpr uint32_t kTfStage = 2 * kTfX + 2 * kTfQ;    // xb (in place of x), xs, qb, qs
constexpr uint32_t kTfLoadBytes = kTfX + 2 * kTfQ;    // TMA bytes per stage
constexpr int kTfThreads = 320;
constexpr uint32_t kTfTmemCols = 32;                  // two 16-column accumulators
constexpr uint32_t kTfIdesc = tc::instr_desc_tf32<kTfM, kTfN>();

NNDEX_DEVICE_INLINE float tf32_head(float v) { return __uint_as_float(__float_as_uint(v) & 0xFFFFE000u); }

NNDEX_DEVICE_INLINE uint8_t* align_1024(uint8_t* p) {
    const uint32_t a = smem_u32(p);
    return p + ((1024u - (a & 1023u)) & 1023u);
}
}  // namespace

size_t tf32_smem_bytes(uint32_t stages, uint32_t cap) {
    size_t b = 1024;                                   // alignment of the swizzled ring
    b += static_cast<size_t>(stages) * kTfStage;
    b += static_cast<size_t>(kTfN) * cap * 8;          // candidate keys
    b += 4 * 256 * 4;                                  // per-warp selection histograms
    b += kTfN * 8 + kTfN * 4;                          // thresholds, counts
    b += (3 * static_cast<size_t>(stages) + 4) * 8 + 16;  // barriers, TMEM slot, abort flag
    return b;
}

template <int ST>
__global__ void __launch_bounds__(kTfThreads, 1)
    scan_tf32_kernel(const __grid_constant__ CUtensorMap tmap_x, const __grid_constant__ CUtensorMap tmap_qb,
                     const __grid_constant__ CUtensorMap tmap_qs, const Tf32ScanArgs p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* ring = align_1024(smem_raw);
    uint64_t* cand = reinterpret_cast<uint64_t*>(ring + static_cast<size_t>(ST) * kTfStage);
    uint32_t* hist = reinterpret_cast<uint32_t*>(cand + static_cast<size_t>(kTfN) * p.cap);
    uint64_t* thr = reinterpret_cast<uint64_t*>(hist + 4 * 256);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(thr + kTfN);
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(cnt + kTfN);
    uint64_t* split_bar = full_bar + ST;
    uint64_t* empty_bar = split_bar + ST;
    uint64_t* tfull = empty_bar + ST;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    volatile uint32_t* abort_flag = tmem_slot + 1;

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t G = gridDim.x, c = blockIdx.x;
    const uint32_t q0 = blockIdx.y * kTfN;
    const uint32_t nqg = (p.nq - q0) < static_cast<uint32_t>(kTfN) ? (p.nq - q0) : static_cast<uint32_t>(kTfN);
    const uint64_t tiles_total = (p.rows + kTfM - 1) / kTfM;
    const uint64_t t_begin = tiles_total * c / G, t_end = tiles_total * (c + 1) / G;
    const uint32_t ntiles = static_cast<uint32_t>(t_end - t_begin);
    const uint64_t row_begin = t_begin * kTfM;
    const uint32_t nbox = p.nbox;

    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&split_bar[s], 128);
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (threadIdx.x < static_cast<uint32_t>(kTfN)) {
        cnt[threadIdx.x] = 0;
        thr[threadIdx.x] = 0ull;
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, kTfTmemCols);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            tma_prefetch_desc(&tmap_x);
            tma_prefetch_desc(&tmap_qb);
            tma_prefetch_desc(&tmap_qs);
            const uint64_t policy = l2_policy_evict_first();  // the base streams once
            uint32_t it = 0;
            bool stop = false;
            for (uint32_t t = 0; t < ntiles && !stop; ++t) {
                const int32_t y = static_cast<int32_t>(row_begin + static_cast<uint64_t>(t) * kTfM);
                for (uint32_t bx = 0; bx < nbox; ++bx) {
                    const uint32_t s = it % ST, u = it / ST;
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
                    uint8_t* st = ring + static_cast<size_t>(s) * kTfStage;
                    mbar_arrive_expect_tx(&full_bar[s], kTfLoadBytes);
                    tma_load_2d_hint(st, &tmap_x, &full_bar[s], static_cast<int32_t>(bx * 32), y, policy);
                    tma_load_2d(st + 2 * kTfX, &tmap_qb, &full_bar[s], static_cast<int32_t>(bx * 32),
                                static_cast<int32_t>(q0));
                    tma_load_2d(st + 2 * kTfX + kTfQ, &tmap_qs, &full_bar[s], static_cast<int32_t>(bx * 32),
                                static_cast<int32_t>(q0));
                    ++it;
                }
            }
            // Drain: every copy has landed, and every arrival the tensor core owes the empty
            // barriers (one commit per consumed stage) has been made, before the CTA may exit.
            const uint32_t used = it < static_cast<uint32_t>(ST) ? it : ST;
            for (uint32_t s = 0; s < used; ++s) {
                const uint32_t uses = (it - s + ST - 1) / ST;
                if (!mbar_wait_bounded(&full_bar[s], (uses - 1) & 1u, kWaitBudgetCycles))
                    record_status(p.status, kStatusTimeout);
                if (!mbar_wait_bounded(&empty_bar[s], (uses - 1) & 1u, kWaitBudgetCycles))
                    record_status(p.status, kStatusTimeout);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            const uint32_t ring0 = smem_u32(ring);
            uint32_t it = 0;
            for (uint32_t t = 0; t < ntiles; ++t) {
                const uint32_t buf = t & 1u, ub = t >> 1;
                if (ub > 0 && !*abort_flag && !mbar_wait_bounded(&tempty[buf], (ub - 1) & 1u, kWaitBudgetCycles)) {
                    *abort_flag = 1;
                    record_status(p.status, kStatusTimeout);
                }
                tc::fence_after_sync();
                const uint32_t d = tmem_base + buf * kTfN;
                for (uint32_t bx = 0; bx < nbox; ++bx, ++it) {
                    const uint32_t s = it % ST, u = it / ST;
                    if (!*abort_flag && !mbar_wait_bounded(&split_bar[s], u & 1u, kWaitBudgetCycles)) {
                        *abort_flag = 1;
                        record_status(p.status, kStatusTimeout);
                    }
                    tc::fence_after_sync();
                    if (!*abort_flag) {
                        const uint32_t xa = ring0 + s * kTfStage, xsa = xa + kTfX;
                        const uint32_t qa = xa + 2 * kTfX, qsa = qa + kTfQ;
#pragma unroll
                        for (uint32_t kk = 0; kk < 4; ++kk) {  // 8 TF32 values (32 bytes) per MMA
                            const uint64_t dx = tc::smem_desc_sw128(xa + kk * 32);
                            const uint64_t dxs = tc::smem_desc_sw128(xsa + kk * 32);
                            const uint64_t dq = tc::smem_desc_sw128(qa + kk * 32);
                            const uint64_t dqs = tc::smem_desc_sw128(qsa + kk * 32);
                            tc::mma_tf32(d, dx, dq, kTfIdesc, (bx | kk) != 0u ? 1u : 0u);
                            tc::mma_tf32(d, dx, dqs, kTfIdesc, 1u);
                            tc::mma_tf32(d, dxs, dq, kTfIdesc, 1u);
                        }
                    }
                    tc::commit(&empty_bar[s]);  // frees the stage once the MMAs above have read it
                }
                tc::commit(&tfull[buf]);  // the tile's accumulator is complete
            }
        }
    } else if (warp < 6) {
        // ---------------- split: x → (xb in place, xs) ----------------
        const uint32_t ts = threadIdx.x - 64;  // 0..127
        uint32_t it = 0;
        for (uint32_t t = 0; t < ntiles; ++t) {
            for (uint32_t bx = 0; bx < nbox; ++bx, ++it) {
                const uint32_t s = it % ST, u = it / ST;
                if (!*abort_flag && !mbar_wait_bounded(&full_bar[s], u & 1u, kWaitBudgetCycles)) {
                    *abort_flag = 1;
                    record_status(p.status, kStatusTimeout);
                }
                if (!*abort_flag) {
                    float4* xv = reinterpret_cast<float4*>(ring + static_cast<size_t>(s) * kTfStage);
                    float4* xs = xv + kTfX / 16;
                    // an elementwise map: the swizzle (a permutation of 16-byte chunks) is kept
#pragma unroll
                    for (uint32_t i = ts; i < kTfX / 16; i += 128) {
                        const float4 v = xv[i];
                        const float4 h = make_float4(tf32_head(v.x), tf32_head(v.y), tf32_head(v.z), tf32_head(v.w));
                        xv[i] = h;
                        xs[i] = make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
                    }
                    fence_proxy_async_smem();  // the generic-proxy writes, visible to the MMA
                }
                mbar_arrive(&split_bar[s]);
            }
        }
    } else {
        // ---------------- epilogue: one base row per thread, 16 queries ----------------
        const uint32_t ew = warp - 6;              // selection slot 0..3
        const uint32_t quarter = warp & 3u;        // the TMEM lanes this warp may read
        const uint32_t lrow = quarter * 32 + lane; // row of the tile
        const uint32_t taddr0 = tmem_base + ((quarter * 32u) << 16);
        for (uint32_t t = 0; t < ntiles; ++t) {
            const uint32_t buf = t & 1u, ub = t >> 1;
            if (!*abort_flag && !mbar_wait_bounded(&tfull[buf], ub & 1u, kWaitBudgetCycles)) {
                *abort_flag = 1;
                record_status(p.status, kStatusTimeout);
            }
            tc::fence_after_sync();
            uint32_t v[16];
            __syncwarp();
            tc::tmem_ld16(taddr0 + buf * kTfN, v);
            tc::tmem_wait_ld16(v);
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[buf]);
            const uint64_t row = row_begin + static_cast<uint64_t>(t) * kTfM + lrow;
            if (row < p.rows && !*abort_flag) {
#pragma unroll
                for (uint32_t j = 0; j < static_cast<uint32_t>(kTfN); ++j) {
                    if (j < nqg) {
                        const uint64_t key = make_key(__uint_as_float(v[j]) + p.eps, static_cast<uint32_t>(row));
                        if (key > thr[j]) {
                            const uint32_t pos = atomicAdd(&cnt[j], 1u);
                            if (pos < p.cap)
                                cand[static_cast<size_t>(j) * p.cap + pos] = key;
                            else
                                record_status(p.status, kStatusOverflow);
                        }
                    }
                }
            }
            named_bar_sync(1, 128);
            scan_flush_g<kTfN, 4, kTfM>(t + 1 == ntiles, nqg, p.kp, p.cap, ew, lane, cnt, thr, cand, hist);
        }
        for (uint32_t b = ew; b < nqg; b += 4) {
            const uint32_t n = cnt[b] < p.kp ? cnt[b] : p.kp;
            uint64_t* dst = p.ws_keys + (static_cast<size_t>(q0 + b) * G + c) * p.kp;
            const uint64_t* src = cand + static_cast<size_t>(b) * p.cap;
            for (uint32_t j = lane; j < p.kp; j += 32) dst[j] = j < n ? src[j] : 0ull;
        }
    }
    // ---------------- teardown: release TMEM ----------------
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem_base, kTfTmemCols);
    }
}

// qb = the TF32 head of each normalised query value, qs = the rest; rows nq..nq_alloc−1 zero.
__global__ void split_queries_tf32_kernel(const float* __restrict__ qn, uint32_t nq, uint32_t ds, uint32_t nq_alloc,
                                          float* __restrict__ qb, float* __restrict__ qs) {
    const size_t n = static_cast<size_t>(nq_alloc) * ds;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t r = static_cast<uint32_t>(i / ds);
        const float v = r < nq ? qn[i] : 0.0f;
        const float h = tf32_head(v);
        qb[i] = h;
        qs[i] = v - h;
    }
}

// Deepest ring (4, 3 or 2 stages) whose footprint fits `smem_limit`; 0 if none.
uint32_t tf32_stages_for(uint32_t cap, size_t smem_limit) {
    for (uint32_t st = 4; st >= 2; --st)
        if (tf32_smem_bytes(st, cap) <= smem_limit) return st;
    return 0;
}

cudaError_t launch_split_queries_tf32(const float* qn, uint32_t nq, uint32_t ds, uint32_t nq_alloc, float* qb,
                                      float* qs, cudaStream_t stream) {
    const size_t n = static_cast<size_t>(nq_alloc) * ds;
    const uint32_t blocks = static_cast<uint32_t>(std::min<size_t>((n + 255) / 256, 1024));
    split_queries_tf32_kernel<<<blocks, 256, 0, stream>>>(qn, nq, ds, nq_alloc, qb, qs);
    count_launch();
    return cudaGetLastError();
}

template <int ST>
static cudaError_t launch_tf32_impl(const CUtensorMap& tx, const CUtensorMap& tqb, const CUtensorMap& tqs,
                                    const Tf32ScanArgs& a, uint32_t ctas, uint32_t qblocks, cudaStream_t stream) {
    auto kern = scan_tf32_kernel<ST>;
    const size_t smem = tf32_smem_bytes(ST, a.cap);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    if (sync_check_enabled())
        set_launch_note("scan_tf32 stages %d: grid (%u, %u), nq %u, k' %u, cap %u, slabs %u, rows %llu, smem %zu", ST,
                        ctas, qblocks, a.nq, a.kp, a.cap, a.nbox, (unsigned long long)a.rows, smem);
    kern<<<dim3(ctas, qblocks), kTfThreads, smem, stream>>>(tx, tqb, tqs, a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_scan_tf32(const CUtensorMap& tx, const CUtensorMap& tqb, const CUtensorMap& tqs,
                             const Tf32ScanArgs& a, uint32_t stages, uint32_t ctas, cudaStream_t stream) {
    const uint32_t qblocks = (a.nq + kTfN - 1) / kTfN;
    if (a.kp == 0 || a.cap < a.kp + kTfM || ctas == 0 || qblocks == 0) return cudaErrorInvalidValue;
    switch (stages) {
        case 4: return launch_tf32_impl<4>(tx, tqb, tqs, a, ctas, qblocks, stream);
        case 3: return launch_tf32_impl<3>(tx, tqb, tqs, a, ctas, qblocks, stream);
        case 2: return launch_tf32_impl<2>(tx, tqb, tqs, a, ctas, qblocks, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace nndex
