// scan_tf32.cu — K12: exact top-k of small query batches from one TF32 tensor-core product per
// (row, query), reranked and certified in FP32.
//
// Replaces the FP32 FMA stream of the exact scan (src/gpu.rs score pass, src/cpu.rs dot loop) where
// that stream, not HBM, bounds it: at 9–16 queries the FP32 scan needs 2·B FLOPs per base byte and
// runs out of issue slots near 60 % of the HBM rate. Here the tensor cores score every staged tile
// straight from the TMA buffer (kind::tf32 reads the FP32 values' sign, exponent and top 10
// mantissa bits), so the CUDA cores only read the accumulators.
//
// s̃ = q̂·x̂ is not the FP32 scan's score, so it only ranks candidates by an upper bound
//   u = s̃ + ε(r, q),   ε = ‖q‖·‖d_x‖ + ‖d_q‖·‖x‖ + ‖d_q‖·‖d_x‖ + C·‖q‖·‖x‖,
// where d_v = v − (v with its 13 low mantissa bits cleared). Whether the tensor core truncates or
// rounds to nearest, |v_i − v̂_i| ≤ |d_v,i|, so the first three terms bound |q·x − q̂·x̂|
// (Cauchy–Schwarz on q·(x − x̂) + (q − q̂)·x̂). C·‖q‖‖x‖ bounds the rest: the tensor core's FP32
// accumulation of ds products (4·ds·2⁻²³ of Σ|q̂_i x̂_i| ≤ ‖q‖‖x‖, the margin the BF16 scan takes),
// the FP32 scan's own rounding ((ds/8 + 3)·2⁻²⁴) and the rounding of u itself (2⁻²²). The norms are
// FP64 sums rounded up: ‖x‖ and ‖d_x‖ per row once per index (row_norms), ‖q‖ and ‖d_q‖ per query
// by the epilogue warps before the first tile.
//
// Each CTA keeps, per query, the k′ rows with the largest u. The merge keeps each query's k′ best,
// and the exact rerank (K4: the FP32 scan's own summation order) returns the top-k with the
// certificate "exact k-th > k′-th bound": every other row's FP32 score is ≤ its u ≤ that bound. So a
// certified query's rows and scores are bit for bit those of the FP32 scan; an uncertified one is
// re-run on the FP32 scan by the host.
//
// Layout: one CTA per (row range, block of 16 queries); ring stages of 128 base rows × one 128-byte
// slab (32 FP32 values) plus the 16 queries' slab, both loaded by TMA with the 128-byte swizzle that
// the MMA's shared-memory descriptors read. The MMA is M = 128 rows × N = 16 queries × K = 8; each
// tile's accumulator is 16 TMEM columns, and eight of them rotate, so the epilogue may fall seven
// tiles behind (a selection) before the tensor core waits. The epilogue thread of TMEM lane r owns
// base row r of the tile: it reads its 16 scores and appends each (u, row) key that beats its
// query's running k′-th key. Selection is the FP32 scan's own machinery (scan_flush_g).
//
// Warps: 0 TMA producer, 1 MMA issuer, 2–5 epilogue. Every wait is bounded; on a timeout the kernel
// records it in the status word, stops issuing, drains its copies and the tensor core's barrier
// arrivals, frees its TMEM and exits.
#include <cuda.h>

#include <algorithm>
#include <cfloat>

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
constexpr uint32_t kTfStage = kTfX + kTfQ;            // 18 KB, a multiple of the 1 KB swizzle atom
constexpr int kTfThreads = 192;
constexpr int kTfAcc = 8;                             // accumulators in flight
constexpr uint32_t kTfTmemCols = 128;                 // kTfAcc × 16 columns
constexpr uint32_t kTfIdesc = tc::instr_desc_tf32<kTfM, kTfN>();

NNDEX_DEVICE_INLINE float tf32_head(float v) { return __uint_as_float(__float_as_uint(v) & 0xFFFFE000u); }

NNDEX_DEVICE_INLINE uint8_t* align_1024(uint8_t* p) {
    const uint32_t a = smem_u32(p);
    return p + ((1024u - (a & 1023u)) & 1023u);
}

// ‖v‖ and ‖v − tf32_head(v)‖ of `n` floats, rounded up, by one warp (FP64 sums).
NNDEX_DEVICE_INLINE float2 warp_tf32_norms(const float* v, uint32_t n, uint32_t lane) {
    double s1 = 0.0, s2 = 0.0;
    for (uint32_t i = lane; i < n; i += 32) {
        const float x = v[i];
        const float d = x - tf32_head(x);  // exact: x and its head share the exponent
        s1 += static_cast<double>(x) * x;
        s2 += static_cast<double>(d) * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, o);
        s2 += __shfl_xor_sync(0xFFFFFFFFu, s2, o);
    }
    return make_float2(__double2float_ru(__dsqrt_ru(s1)), __double2float_ru(__dsqrt_ru(s2)));
}
}  // namespace

size_t tf32_smem_bytes(uint32_t stages, uint32_t cap) {
    size_t b = 1024;                                   // alignment of the swizzled ring
    b += static_cast<size_t>(stages) * kTfStage;
    b += static_cast<size_t>(kTfN) * cap * 8;          // candidate keys
    b += 4 * 256 * 4;                                  // per-warp selection histograms
    b += kTfN * 8 + kTfN * 4 + kTfN * 8;               // thresholds, counts, query norms
    b += (2 * static_cast<size_t>(stages) + 2 * kTfAcc) * 8 + 16;  // barriers, TMEM slot, abort flag
    return b;
}

template <int ST>
__global__ void __launch_bounds__(kTfThreads, 1)
    scan_tf32_kernel(const __grid_constant__ CUtensorMap tmap_x, const __grid_constant__ CUtensorMap tmap_q,
                     const Tf32ScanArgs p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* ring = align_1024(smem_raw);
    uint64_t* cand = reinterpret_cast<uint64_t*>(ring + static_cast<size_t>(ST) * kTfStage);
    uint32_t* hist = reinterpret_cast<uint32_t*>(cand + static_cast<size_t>(kTfN) * p.cap);
    uint64_t* thr = reinterpret_cast<uint64_t*>(hist + 4 * 256);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(thr + kTfN);
    float2* qnorm = reinterpret_cast<float2*>(cnt + kTfN);
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(qnorm + kTfN);
    uint64_t* empty_bar = full_bar + ST;
    uint64_t* tfull = empty_bar + ST;
    uint64_t* tempty = tfull + kTfAcc;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + kTfAcc);
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
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < kTfAcc; ++b) {
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
            tma_prefetch_desc(&tmap_q);
            // the base streams once unless several query blocks read the same rows
            const uint64_t policy = p.evict_first ? l2_policy_evict_first() : l2_policy_evict_normal();
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
                    mbar_arrive_expect_tx(&full_bar[s], kTfStage);
                    tma_load_2d_hint(st, &tmap_x, &full_bar[s], static_cast<int32_t>(bx * 32), y, policy);
                    tma_load_2d(st + kTfX, &tmap_q, &full_bar[s], static_cast<int32_t>(bx * 32),
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
                const uint32_t buf = t % kTfAcc, ub = t / kTfAcc;
                if (ub > 0 && !*abort_flag && !mbar_wait_bounded(&tempty[buf], (ub - 1) & 1u, kWaitBudgetCycles)) {
                    *abort_flag = 1;
                    record_status(p.status, kStatusTimeout);
                }
                tc::fence_after_sync();
                const uint32_t d = tmem_base + buf * kTfN;
                for (uint32_t bx = 0; bx < nbox; ++bx, ++it) {
                    const uint32_t s = it % ST, u = it / ST;
                    if (!*abort_flag && !mbar_wait_bounded(&full_bar[s], u & 1u, kWaitBudgetCycles)) {
                        *abort_flag = 1;
                        record_status(p.status, kStatusTimeout);
                    }
                    tc::fence_after_sync();
                    if (!*abort_flag) {
                        const uint32_t xa = ring0 + s * kTfStage, qa = xa + kTfX;
#pragma unroll
                        for (uint32_t kk = 0; kk < 4; ++kk)  // 8 TF32 values (32 bytes) per MMA
                            tc::mma_tf32(d, tc::smem_desc_sw128(xa + kk * 32), tc::smem_desc_sw128(qa + kk * 32),
                                         kTfIdesc, (bx | kk) != 0u ? 1u : 0u);
                    }
                    tc::commit(&empty_bar[s]);  // frees the stage once the MMAs above have read it
                }
                tc::commit(&tfull[buf]);  // the tile's accumulator is complete
            }
        }
    } else {
        // ---------------- epilogue: one base row per thread, 16 queries ----------------
        const uint32_t ew = warp - 2;              // selection slot 0..3
        const uint32_t quarter = warp & 3u;        // the TMEM lanes this warp may read
        const uint32_t lrow = quarter * 32 + lane; // row of the tile
        const uint32_t taddr0 = tmem_base + ((quarter * 32u) << 16);
        for (uint32_t j = ew; j < nqg; j += 4) {
            const float2 n = warp_tf32_norms(p.queries + static_cast<size_t>(q0 + j) * p.ds, p.ds, lane);
            if (lane == 0) qnorm[j] = n;
        }
        named_bar_sync(1, 128);
        const float cn = p.c_norm;
        for (uint32_t t = 0; t < ntiles; ++t) {
            const uint32_t buf = t % kTfAcc, ub = t / kTfAcc;
            const uint64_t row = row_begin + static_cast<uint64_t>(t) * kTfM + lrow;
            const float2 rn = row < p.rows ? p.row_norms[row] : make_float2(0.0f, 0.0f);
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
            if (row < p.rows && !*abort_flag) {
                // ε = ‖q‖·(‖d_x‖ + C‖x‖) + ‖d_q‖·(‖x‖ + ‖d_x‖), with 1 % for its own roundings
                const float P = fmaf(cn, rn.x, rn.y), Q = rn.x + rn.y;
#pragma unroll
                for (uint32_t j = 0; j < static_cast<uint32_t>(kTfN); ++j) {
                    if (j < nqg) {
                        const float2 qq = qnorm[j];
                        const float eps = fmaf(qq.x, P, qq.y * Q) * 1.01f;
                        float u = __uint_as_float(v[j]) + eps;
                        if (!(u <= FLT_MAX)) u = INFINITY;  // an overflowing or NaN bound keeps the row
                        const uint64_t key = make_key(u, static_cast<uint32_t>(row));
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
            unsigned long long mn = ~0ull;
            for (uint32_t j = lane; j < p.kp; j += 32) {
                const uint64_t key = j < n ? src[j] : 0ull;
                dst[j] = key;
                mn = key < mn ? key : mn;
            }
            if (p.floor_keys && n == p.kp) {  // a full list: every row it left out has a smaller key
#pragma unroll
                for (uint32_t o = 16; o > 0; o >>= 1) {
                    const unsigned long long x = __shfl_xor_sync(0xFFFFFFFFu, mn, o);
                    mn = x < mn ? x : mn;
                }
                if (lane == 0) atomicMax(&p.floor_keys[q0 + b], mn);
            }
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

// Per row of the base: {‖x‖, ‖x − tf32_head(x)‖}, rounded up (one warp per row).
__global__ void tf32_row_norms_kernel(const float* __restrict__ base, uint64_t rows, uint32_t ds,
                                      float2* __restrict__ out) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w0 = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t r = w0; r < rows; r += nw) {
        const float2 n = warp_tf32_norms(base + r * ds, ds, lane);
        if (lane == 0) out[r] = n;
    }
}

cudaError_t launch_tf32_row_norms(const float* base, uint64_t rows, uint32_t ds, float2* out, uint32_t sm_count,
                                  cudaStream_t stream) {
    if (rows == 0) return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>((rows + 7) / 8, static_cast<uint64_t>(sm_count) * 8);
    tf32_row_norms_kernel<<<static_cast<uint32_t>(blocks), 256, 0, stream>>>(base, rows, ds, out);
    count_launch();
    return cudaGetLastError();
}

// Deepest ring (8 down to 2 stages) whose footprint fits `smem_limit`; 0 if none.
uint32_t tf32_stages_for(uint32_t cap, size_t smem_limit) {
    for (uint32_t st = 8; st >= 2; --st)
        if (tf32_smem_bytes(st, cap) <= smem_limit) return st;
    return 0;
}

template <int ST>
static cudaError_t launch_tf32_impl(const CUtensorMap& tx, const CUtensorMap& tq, const Tf32ScanArgs& a,
                                    uint32_t ctas, uint32_t qblocks, cudaStream_t stream) {
    auto kern = scan_tf32_kernel<ST>;
    const size_t smem = tf32_smem_bytes(ST, a.cap);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    if (sync_check_enabled())
        set_launch_note("scan_tf32 stages %d: grid (%u, %u), nq %u, k' %u, cap %u, slabs %u, rows %llu, smem %zu", ST,
                        ctas, qblocks, a.nq, a.kp, a.cap, a.nbox, (unsigned long long)a.rows, smem);
    kern<<<dim3(ctas, qblocks), kTfThreads, smem, stream>>>(tx, tq, a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_scan_tf32(const CUtensorMap& tx, const CUtensorMap& tq, const Tf32ScanArgs& a, uint32_t stages,
                             uint32_t ctas, cudaStream_t stream) {
    const uint32_t qblocks = (a.nq + kTfN - 1) / kTfN;
    if (a.kp == 0 || a.cap < a.kp + kTfM || ctas == 0 || qblocks == 0 || !a.queries || !a.row_norms)
        return cudaErrorInvalidValue;
    switch (stages) {
        case 8: return launch_tf32_impl<8>(tx, tq, a, ctas, qblocks, stream);
        case 7: return launch_tf32_impl<7>(tx, tq, a, ctas, qblocks, stream);
        case 6: return launch_tf32_impl<6>(tx, tq, a, ctas, qblocks, stream);
        case 5: return launch_tf32_impl<5>(tx, tq, a, ctas, qblocks, stream);
        case 4: return launch_tf32_impl<4>(tx, tq, a, ctas, qblocks, stream);
        case 3: return launch_tf32_impl<3>(tx, tq, a, ctas, qblocks, stream);
        case 2: return launch_tf32_impl<2>(tx, tq, a, ctas, qblocks, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace nndex
