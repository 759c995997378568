// ivf_build.cu — K5-K7: the IVF build of nndex's approximate mode on the GPU.
//
// Replaces ApproxIndex::build (src/approx.rs:46-100): medoid (409-429), k-means++ seeding
// (357-406), spherical k-means (434-535) and the cluster-contiguous reorder. The result is the
// reference's index bit for bit (same seeds, centroids, assignments, list order), so searches over
// it probe the same lists. Every decision the reference takes on a simsimd f32 dot (FP64
// accumulation of f32 products, rounded to f32 — src/approx.rs:539-552) is taken here on the same
// value: products of two f32 are exact in FP64, and the sum is accumulated in index order.
//
// Where the time goes and how it is spent on B200:
//   * seeding: nlist − 1 sequential passes over the rows. Each pass screens every row with an FP16
//     dot (half the bytes of FP32) and a rigorous error bound; only rows whose distance could drop
//     below their running minimum are re-scored exactly (FP64 sequential dot). The running sum of
//     the minima and the threshold search are exact: every distance is a multiple of 2^-24, so FP64
//     sums below 2^29 carry no rounding and any summation order gives the reference's value.
//   * assignment: a tcgen05 FP16 GEMM rows × centroids (M = 128 rows in TMEM lanes, N = 256
//     centroids), run twice. Pass A keeps each row's best approximate score s1. Pass B repeats the
//     GEMM and lists every centroid whose approximate score reaches s1 − 2e (e = the row's error
//     bound); every other centroid scores strictly lower, exactly. A row with one listed centroid
//     is assigned to it; a row with at most 32 is decided by one warp with exact FP64 dots against
//     those candidates (highest f32 score, lowest index on a tie: the reference's strict `>` in
//     index order); a row with more, or with a non-finite bound, is re-scored exactly against every
//     centroid.
//     FP16 (11-bit significand) suits unit rows and centroids: its error bound is 8× tighter than
//     BF16's. Values in FP16's subnormal range count as lost in the residual, so the bound holds
//     whether the tensor core keeps or flushes them; an overflow makes the bound infinite (or NaN),
//     which sends the row to the exact pass.
//   * update: a stable counting sort by cluster (row order kept inside each cluster) and FP64 sums
//     in that order — the reference's summation order — then the reference's normalisation, each
//     operation rounded as in Rust (no contraction).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "index.h"
#include "internal.h"
#include "ivf.h"
#include "select.cuh"
#include "tc.cuh"

namespace nndex {

bool encode_tmap_2d(CUtensorMap* map, CUtensorMapDataType dtype, uint32_t elem_bytes, const void* base,
                    uint64_t inner, uint64_t outer, uint64_t row_stride_bytes, uint32_t box_inner,
                    uint32_t box_outer, CUtensorMapSwizzle swizzle);

namespace {

NNDEX_DEVICE_INLINE uint8_t* align_1024(uint8_t* p) {
    const uint32_t a = smem_u32(p);
    return p + ((1024u - (a & 1023u)) & 1023u);
}

// f32 with −0 folded into +0: the reference compares scores with `>` on f32, where −0 == +0.
NNDEX_DEVICE_INLINE float fold_zero(float f) { return f == 0.0f ? 0.0f : f; }

// The reference's dot_small / simsimd f32 dot on n ≥ 8 values: FP64 accumulation in index order of
// exact f32 × f32 products, rounded to f32 (src/approx.rs:539-552). fma(a, b, s) rounds once, like
// s + a·b with an exact product.
NNDEX_DEVICE_INLINE float dot_f64_seq(const float* __restrict__ x, const float* __restrict__ y, uint32_t n) {
    double s = 0.0;
    uint32_t d = 0;
    for (; d + 4 <= n; d += 4) {
        const float4 a = *reinterpret_cast<const float4*>(x + d);
        const float4 b = *reinterpret_cast<const float4*>(y + d);
        s = fma(static_cast<double>(a.x), static_cast<double>(b.x), s);
        s = fma(static_cast<double>(a.y), static_cast<double>(b.y), s);
        s = fma(static_cast<double>(a.z), static_cast<double>(b.z), s);
        s = fma(static_cast<double>(a.w), static_cast<double>(b.w), s);
    }
    for (; d < n; ++d) s = fma(static_cast<double>(x[d]), static_cast<double>(y[d]), s);
    return __double2float_rn(s);
}

// Same with the second operand dims-major (column c of a [n × stride] matrix).
NNDEX_DEVICE_INLINE float dot_f64_seq_col(const float* __restrict__ x, const float* __restrict__ ct, uint64_t stride,
                                          uint32_t c, uint32_t n) {
    double s = 0.0;
    for (uint32_t d = 0; d < n; ++d)
        s = fma(static_cast<double>(x[d]), static_cast<double>(ct[static_cast<uint64_t>(d) * stride + c]), s);
    return __double2float_rn(s);
}

NNDEX_DEVICE_INLINE double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// FP16 copy of v, and the residual the error bounds use: v − half(v) when half(v) is a normal FP16
// value; a value in the subnormal range (or zero) counts as entirely lost.
NNDEX_DEVICE_INLINE __half to_f16(float v, float& resid) {
    const __half h = __float2half_rn(v);
    const float hf = __half2float(h);
    resid = fabsf(hf) >= 6.103515625e-05f ? v - hf : v;  // 2^-14: the smallest normal FP16
    return h;
}

// Upper bound of sqrt(v) as f32 for v ≥ 0 accumulated in FP64 (relative slack for its rounding).
NNDEX_DEVICE_INLINE float sqrt_up(double v) {
    return __double2float_ru(__dsqrt_ru(v * (1.0 + 1e-12)));
}

}  // namespace

// ------------------------------------------------------------------------------------------
// Row preparation: FP16 copy and per row upper bounds of ‖x‖ and of the residual ‖x − x̂‖. One
// warp per row.
// ------------------------------------------------------------------------------------------
__global__ void ivf_row_prep_kernel(const float* __restrict__ src, uint32_t ds, uint64_t rows,
                                    __half* __restrict__ out16, uint32_t kb, float* __restrict__ norm_up,
                                    float* __restrict__ res_up) {
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t r = warp; r < rows; r += nwarps) {
        const float* x = src + r * ds;
        double n2 = 0.0, r2 = 0.0;
        for (uint32_t d = lane; d < kb; d += 32) {
            const float v = d < ds ? x[d] : 0.0f;
            float e;
            const __half b = to_f16(v, e);
            n2 = fma(static_cast<double>(v), static_cast<double>(v), n2);
            r2 = fma(static_cast<double>(e), static_cast<double>(e), r2);
            out16[r * kb + d] = b;
        }
        n2 = warp_sum_d(n2);
        r2 = warp_sum_d(r2);
        if (lane == 0) {
            norm_up[r] = sqrt_up(n2);
            res_up[r] = sqrt_up(r2);
        }
    }
}

// ------------------------------------------------------------------------------------------
// Medoid (src/approx.rs:409-429). Column sums in row order, FP64: one warp per 32 columns, the
// rows staged through shared memory by TMA (128-row boxes of 128 bytes, 128-byte swizzle) in an
// 8-deep ring; lane = column. Then mean_f32[d] = (sum · (1/rows)) as f32.
// ------------------------------------------------------------------------------------------
namespace {
constexpr int kColStages = 8;
constexpr uint32_t kColStageBytes = 128 * 128;
}  // namespace

__global__ void __launch_bounds__(64, 1)
    colsum_mean_kernel(const __grid_constant__ CUtensorMap tmap, uint64_t rows, float* __restrict__ mean_f32,
                       uint32_t* __restrict__ status) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* ring = align_1024(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + kColStages * kColStageBytes);
    uint64_t* empty = full + kColStages;
    volatile uint32_t* abort_flag = reinterpret_cast<volatile uint32_t*>(empty + kColStages);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t box = blockIdx.x;  // 32-column slab
    const uint32_t ntiles = static_cast<uint32_t>((rows + 127) / 128);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kColStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    if (warp == 0) {
        if (lane == 0) {
            uint32_t t = 0;
            for (; t < ntiles; ++t) {
                const uint32_t s = t % kColStages, u = t / kColStages;
                if (u > 0 && !mbar_wait_bounded(&empty[s], (u - 1) & 1u, kWaitBudgetCycles)) {
                    *abort_flag = 1;
                    record_status(status, kStatusTimeout);
                    break;
                }
                if (*abort_flag) break;
                mbar_arrive_expect_tx(&full[s], kColStageBytes);
                tma_load_2d(ring + s * kColStageBytes, &tmap, &full[s], static_cast<int32_t>(box * 32),
                            static_cast<int32_t>(t * 128));
            }
            const uint32_t used = t < static_cast<uint32_t>(kColStages) ? t : kColStages;
            for (uint32_t s = 0; s < used; ++s) {
                const uint32_t uses = (t - s + kColStages - 1) / kColStages;
                if (!mbar_wait_bounded(&full[s], (uses - 1) & 1u, kWaitBudgetCycles)) record_status(status, kStatusTimeout);
            }
        }
        return;
    }
    double sum = 0.0;
    const uint32_t chunk = lane >> 2, within = (lane & 3u) * 4;
    for (uint32_t t = 0; t < ntiles; ++t) {
        const uint32_t s = t % kColStages, u = t / kColStages;
        if (*abort_flag || !mbar_wait_bounded(&full[s], u & 1u, kWaitBudgetCycles)) {
            *abort_flag = 1;
            record_status(status, kStatusTimeout);
            break;
        }
        const uint8_t* st = ring + s * kColStageBytes;
        const uint32_t nr = (rows - static_cast<uint64_t>(t) * 128) < 128 ? static_cast<uint32_t>(rows - t * 128ull) : 128u;
        for (uint32_t r = 0; r < nr; ++r) {
            const float v =
                *reinterpret_cast<const volatile float*>(st + r * 128 + ((chunk ^ (r & 7u)) * 16) + within);
            sum = __dadd_rn(sum, static_cast<double>(v));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
    const double inv_rows = __ddiv_rn(1.0, static_cast<double>(rows));
    mean_f32[box * 32 + lane] = __double2float_rn(__dmul_rn(sum, inv_rows));
}

// argmax over rows of dot_small(row, mean) — the first strict maximum, i.e. the largest key.
__global__ void medoid_kernel(const float* __restrict__ base, uint32_t ds, uint32_t dp, uint64_t rows,
                              const float* __restrict__ mean_f32, unsigned long long* __restrict__ best) {
    extern __shared__ float mean_s[];
    for (uint32_t d = threadIdx.x; d < ds; d += blockDim.x) mean_s[d] = mean_f32[d];
    __syncthreads();
    unsigned long long bk = 0;
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < rows;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float s = fold_zero(dot_f64_seq(base + r * ds, mean_s, dp));
        const unsigned long long key = make_key(s, static_cast<uint32_t>(r));
        bk = key > bk ? key : bk;
    }
    bk = warp_max_u64(bk);
    if ((threadIdx.x & 31u) == 0) atomicMax(best, bk);
}

// ------------------------------------------------------------------------------------------
// k-means++ seeding step c (src/approx.rs:370-402): min_d[r] = min(min_d[r], max(1 − dot(r, c−1),
// 0)); total = Σ min_d; the LCG draws a threshold; the chosen row is the first whose running sum
// reaches it. One launch per centroid; the last block to finish does the draw and the search.
// ------------------------------------------------------------------------------------------
struct KppState {
    unsigned long long rng;
    unsigned int done;
    unsigned int pad;
    unsigned long long exact_rows;
};

namespace {
constexpr uint32_t kKppThreads = 256;
constexpr uint32_t kKppScanChunk = 2048;
}  // namespace

__global__ void __launch_bounds__(kKppThreads)
    kpp_step_kernel(const float* __restrict__ base, const __half* __restrict__ b16, uint32_t ds, uint32_t kb,
                    uint32_t dp, uint64_t rows, uint64_t rows_per_block, const float* __restrict__ norm_up,
                    const float* __restrict__ res_up, float gamma, float* __restrict__ min_d,
                    double* __restrict__ partial, KppState* __restrict__ st, uint32_t* __restrict__ chosen,
                    uint32_t c) {
    extern __shared__ uint8_t smem_raw[];
    float* cf = reinterpret_cast<float*>(smem_raw);                        // ds
    __half* cb = reinterpret_cast<__half*>(cf + ds);                      // kb
    float* scan_buf = reinterpret_cast<float*>(cb + kb);                   // kKppScanChunk (last block)
    __shared__ double wsum[kKppThreads / 32];
    __shared__ unsigned int is_last;
    __shared__ double sh_total, sh_thr, sh_before;
    __shared__ unsigned long long sh_blk;
    __shared__ unsigned int sh_found;
    __shared__ unsigned long long sh_exact;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t prev = chosen[c - 1];
    for (uint32_t d = tid; d < ds; d += blockDim.x) cf[d] = base[static_cast<uint64_t>(prev) * ds + d];
    for (uint32_t d = tid; d < kb; d += blockDim.x) cb[d] = b16[static_cast<uint64_t>(prev) * kb + d];
    if (tid == 0) sh_exact = 0;
    __syncthreads();
    const float nc = norm_up[prev], rc = res_up[prev];
    const uint64_t r0 = static_cast<uint64_t>(blockIdx.x) * rows_per_block;
    const uint64_t r1 = (r0 + rows_per_block) < rows ? (r0 + rows_per_block) : rows;
    const uint32_t g = lane >> 3, j = lane & 7u;  // 4 rows per warp, 8 lanes per row
    const uint32_t nch = kb / 8;                    // 16-byte chunks of a BF16 row
    double acc = 0.0;
    uint32_t exact_here = 0;
    const uint4* cr = reinterpret_cast<const uint4*>(cb);
    for (uint64_t rb = r0 + warp * 4; rb < r1; rb += (kKppThreads / 32) * 4) {
        const uint64_t r = rb + g;
        const bool live = r < r1;
        // Every load of the row first (its FP16 chunks; lane 0 of the group: min_d and the row's
        // bounds), so a row costs one memory round trip.
        float m = 0.0f, nr = 0.0f, rr = 0.0f;
        if (live && j == 0) {
            m = min_d[r];
            nr = norm_up[r];
            rr = res_up[r];
        }
        constexpr int kPre = 8;  // chunks per lane in flight (rows up to 512 FP16 values)
        const uint4* xr = reinterpret_cast<const uint4*>(b16 + (live ? r : r0) * kb);
        uint4 xa[kPre];
#pragma unroll
        for (int u = 0; u < kPre; ++u) {
            const uint32_t ch = j + 8u * u;
            xa[u] = (live && ch < nch) ? xr[ch] : make_uint4(0u, 0u, 0u, 0u);
        }
        float sd = 0.0f;
        auto dot_chunk = [&](const uint4& a, const uint4& b) {
            const __half2* a2 = reinterpret_cast<const __half2*>(&a);
            const __half2* b2 = reinterpret_cast<const __half2*>(&b);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float2 fa = __half22float2(a2[i]), fb = __half22float2(b2[i]);
                sd = fmaf(fa.x, fb.x, sd);
                sd = fmaf(fa.y, fb.y, sd);
            }
        };
#pragma unroll
        for (int u = 0; u < kPre; ++u) {
            const uint32_t ch = j + 8u * u;
            if (ch < nch) dot_chunk(xa[u], cr[ch]);
        }
        if (live)
            for (uint32_t ch = j + 8u * kPre; ch < nch; ch += 8) dot_chunk(xr[ch], cr[ch]);
        sd += __shfl_xor_sync(0xffffffffu, sd, 1);
        sd += __shfl_xor_sync(0xffffffffu, sd, 2);
        sd += __shfl_xor_sync(0xffffffffu, sd, 4);
        if (live && j == 0) {
            bool need = m > 0.0f;
            if (need && m < FLT_MAX) {
                // |x·c − x̂·ĉ| ≤ ‖δx‖‖c‖ + ‖x̂‖‖δc‖; + FP32 accumulation of the screen; + the f32
                // rounding of the exact dot and of 1 − dot.
                const float xh = nr + rr, chn = nc + rc;
                const float e = (rr * nc + xh * rc + gamma * xh * chn + 2.4e-7f * fmaxf(1.0f, nr * nc)) * 1.001f;
                const double lb = 1.0 - (static_cast<double>(sd) + static_cast<double>(e));
                need = !(static_cast<double>(m) <= lb);  // a NaN bound (overflowed copy) scores exactly
            }
            if (need) {
                const float dot = dot_f64_seq(base + r * ds, cf, dp);
                const float dist = fmaxf(1.0f - dot, 0.0f);  // (1.0 - dot).max(0.0) in f32
                if (dist < m) {
                    m = dist;
                    min_d[r] = m;
                }
                ++exact_here;
            }
            acc += static_cast<double>(m);
        }
    }
    __threadfence();  // this thread's min_d writes, before the block's ticket below
    acc = warp_sum_d(acc);
    if (lane == 0) wsum[warp] = acc;
    if (exact_here) atomicAdd(&sh_exact, static_cast<unsigned long long>(exact_here));
    __syncthreads();
    if (tid == 0) {
        double b = 0.0;
        for (uint32_t w = 0; w < kKppThreads / 32; ++w) b += wsum[w];
        partial[blockIdx.x] = b;  // exact: a sum of multiples of 2^-24 below 2^29
        atomicAdd(&st->exact_rows, sh_exact);
        __threadfence();
        is_last = (atomicAdd(&st->done, 1u) == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // ---- last block: total, threshold, chosen row ----
    const uint32_t nb = gridDim.x;
    if (warp == 0) {
        double t = 0.0;
        for (uint32_t b = lane; b < nb; b += 32) t += __ldcg(&partial[b]);
        t = warp_sum_d(t);
        if (lane == 0) sh_total = t;
    }
    __syncthreads();
    const double total = sh_total;
    if (total <= 0.0) {
        if (tid == 0) {
            chosen[c] = prev;  // duplicate of the previous centroid; the LCG does not advance
            st->done = 0;
        }
        return;
    }
    if (warp == 0) {
        const unsigned long long rng = st->rng * 6364136223846793005ull + 1ull;
        const double thr = __dmul_rn(__ddiv_rn(__ull2double_rn(rng), __ull2double_rn(~0ull)), total);
        // First block whose running sum reaches thr (sums are exact, so this is the row-order scan).
        double before = 0.0;
        unsigned long long blk = nb;  // none
        for (uint32_t b0 = 0; b0 < nb && blk == nb; b0 += 32) {
            const double v = (b0 + lane < nb) ? __ldcg(&partial[b0 + lane]) : 0.0;
            double incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double n = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= static_cast<uint32_t>(o)) incl += n;
            }
            const unsigned hit = __ballot_sync(0xffffffffu, (b0 + lane < nb) && (before + incl >= thr));
            if (hit) {
                const int l = __ffs(hit) - 1;
                blk = b0 + l;
                before += __shfl_sync(0xffffffffu, incl - v, l);
            } else {
                before += __shfl_sync(0xffffffffu, incl, 31);
            }
        }
        if (lane == 0) {
            st->rng = rng;
            sh_thr = thr;
            sh_before = before;
            sh_blk = blk;
            sh_found = 0;
        }
    }
    __syncthreads();
    uint64_t chosen_row = rows - 1;
    if (sh_blk < nb) {
        const uint64_t b0 = sh_blk * rows_per_block;
        const uint64_t b1 = (b0 + rows_per_block) < rows ? (b0 + rows_per_block) : rows;
        double before = sh_before;
        for (uint64_t s0 = b0; s0 < b1; s0 += kKppScanChunk) {
            const uint32_t n = static_cast<uint32_t>((b1 - s0) < kKppScanChunk ? (b1 - s0) : kKppScanChunk);
            for (uint32_t i = tid; i < n; i += blockDim.x) scan_buf[i] = __ldcg(&min_d[s0 + i]);
            __syncthreads();
            if (warp == 0) {
                for (uint32_t i0 = 0; i0 < n; i0 += 32) {
                    const double v = (i0 + lane < n) ? static_cast<double>(scan_buf[i0 + lane]) : 0.0;
                    double incl = v;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const double nn = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= static_cast<uint32_t>(o)) incl += nn;
                    }
                    const unsigned hit = __ballot_sync(0xffffffffu, (i0 + lane < n) && (before + incl >= sh_thr));
                    if (hit) {
                        if (lane == 0) {
                            sh_found = 1;
                            sh_blk = s0 + i0 + (__ffs(hit) - 1);  // reuse: the chosen row
                        }
                        break;
                    }
                    before += __shfl_sync(0xffffffffu, incl, 31);
                }
            }
            __syncthreads();
            if (sh_found) break;
        }
        if (sh_found) chosen_row = sh_blk;
    }
    if (tid == 0) {
        chosen[c] = static_cast<uint32_t>(chosen_row);
        st->done = 0;
    }
}

__global__ void fill_f32_kernel(float* __restrict__ p, uint64_t n, float v) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        p[i] = v;
}

// BF16 copy of FP32 rows (round to nearest, as the index's own BF16 copy) with an upper bound of
// each row's residual norm ‖x − bf16(x)‖. One warp per row.
__global__ void bf16_rows_kernel(const float* __restrict__ src, uint32_t ds, uint64_t rows, __nv_bfloat16* __restrict__ out,
                                 uint32_t kb, float* __restrict__ res_up) {
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t r = warp; r < rows; r += nwarps) {
        double r2 = 0.0;
        for (uint32_t d = lane; d < kb; d += 32) {
            const float v = d < ds ? src[r * ds + d] : 0.0f;
            const __nv_bfloat16 b = __float2bfloat16_rn(v);
            const float e = v - __bfloat162float(b);  // exact: the rounding residual
            r2 = fma(static_cast<double>(e), static_cast<double>(e), r2);
            out[r * kb + d] = b;
        }
        r2 = warp_sum_d(r2);
        if (lane == 0) res_up[r] = sqrt_up(r2);
    }
}

// Rows → centroid slots (the seeded centroids are copies of rows).
__global__ void gather_rows_kernel(const float* __restrict__ src, uint32_t ds, const uint32_t* __restrict__ idx,
                                   uint64_t n, float* __restrict__ dst) {
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t i = warp; i < n; i += nwarps) {
        const float4* a = reinterpret_cast<const float4*>(src + static_cast<uint64_t>(idx[i]) * ds);
        float4* b = reinterpret_cast<float4*>(dst + i * ds);
        for (uint32_t v = lane; v < ds / 4; v += 32) b[v] = a[v];
    }
}

// ------------------------------------------------------------------------------------------
// Centroid preparation for one assignment: FP16 copy (rows ≥ nlist stay zero), dims-major FP32
// copy, and the largest ‖c‖ and ‖c − ĉ‖ (upper bounds, as f32 bits; non-negative floats order as
// unsigned integers; a NaN bound compares above every finite one). One warp per centroid.
// ------------------------------------------------------------------------------------------
__global__ void centroid_prep_kernel(const float* __restrict__ cent, uint32_t ds, uint32_t nlist,
                                     __half* __restrict__ c16, uint32_t kb, float* __restrict__ cent_t,
                                     uint64_t ct_stride, unsigned int* __restrict__ cmax) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (warp >= nlist) return;
    const float* x = cent + static_cast<uint64_t>(warp) * ds;
    double n2 = 0.0, r2 = 0.0;
    for (uint32_t d = lane; d < kb; d += 32) {
        const float v = d < ds ? x[d] : 0.0f;
        float e;
        const __half b = to_f16(v, e);
        n2 = fma(static_cast<double>(v), static_cast<double>(v), n2);
        r2 = fma(static_cast<double>(e), static_cast<double>(e), r2);
        if (c16) c16[static_cast<uint64_t>(warp) * kb + d] = b;
        if (cent_t && d < ds) cent_t[static_cast<uint64_t>(d) * ct_stride + warp] = v;
    }
    n2 = warp_sum_d(n2);
    r2 = warp_sum_d(r2);
    if (lane == 0 && cmax) {
        atomicMax(&cmax[0], __float_as_uint(sqrt_up(n2)));
        atomicMax(&cmax[1], __float_as_uint(sqrt_up(r2)));
    }
}

// ------------------------------------------------------------------------------------------
// K5: assignment on the tensor cores. Persistent CTAs walk 128-row tiles; for each, every
// 256-centroid tile is one M=128 × N=256 BF16 GEMM (K in 64-element slabs, A and B slabs staged
// together by TMA, 4-deep ring) into one of two TMEM accumulators; the epilogue keeps per row the
// best approximate score (and its centroid) and the second best. Certified rows are assigned;
// the others are queued for the exact pass.
// ------------------------------------------------------------------------------------------
namespace {
constexpr int kAsM = 128;
constexpr int kAsN = 256;
constexpr uint32_t kAsA = kAsM * 128;
constexpr uint32_t kAsB = kAsN * 128;
constexpr uint32_t kAsStage = kAsA + kAsB;
constexpr int kAsStages = 4;
constexpr uint32_t kAsThreads = 192;
constexpr uint32_t kAsTmemCols = 512;
constexpr size_t kAsSmem = 1024 + kAsStages * kAsStage + (2 * kAsStages + 4) * 8 + 16;
constexpr uint32_t kCandCap = 32;  // candidates a row may keep (one warp lane each)

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
}  // namespace

struct AssignParams {
    uint64_t rows = 0;
    uint32_t nlist = 0;
    uint32_t nct = 0;       // centroid tiles of 256
    uint32_t nchunks = 0;   // 64-element K slabs
    const float* norm_up = nullptr;
    const float* res_up = nullptr;
    const unsigned int* cmax = nullptr;  // max ‖c‖, max ‖δc‖ (f32 bits)
    float gamma = 0.0f;                  // FP32 accumulation bound factor
    float* smax = nullptr;          // pass A output: the best approximate score of each row
    uint32_t* assign = nullptr;
    uint32_t* amb = nullptr;        // rows re-scored against every centroid
    uint32_t* amb_cnt = nullptr;
    uint32_t* cand_list = nullptr;  // rows × kCandCap: the centroids inside a row's window
    uint2* cand = nullptr;          // (row, candidates) of the rows decided among their candidates
    uint32_t* cand_cnt = nullptr;
    uint32_t* status = nullptr;
};

// kMode 0 (pass A): each row's best approximate score s1 → smax. kMode 1 (pass B): the same GEMM;
// every centroid whose approximate score reaches s1 − 2e is a candidate (any other scores strictly
// lower than the best, exactly). One candidate: assigned. Up to kCandCap: queued for the exact
// decision among them. More (or a non-finite bound): queued for the all-centroid exact pass.
template <int kMode>
__global__ void __launch_bounds__(kAsThreads, 1)
    kmeans_assign_tc_kernel(const __grid_constant__ CUtensorMap tmap_rows, const __grid_constant__ CUtensorMap tmap_cent,
                            const AssignParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* ring = align_1024(smem_raw);
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(ring + kAsStages * kAsStage);
    uint64_t* empty_bar = full_bar + kAsStages;
    uint64_t* tfull = empty_bar + kAsStages;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    volatile uint32_t* abort_flag = tmem_slot + 1;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t nrt = static_cast<uint32_t>((p.rows + kAsM - 1) / kAsM);
    const uint32_t nct = p.nct, nchunks = p.nchunks;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kAsStages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, kAsTmemCols);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            tma_prefetch_desc(&tmap_rows);
            tma_prefetch_desc(&tmap_cent);
            uint32_t it = 0;
            bool stop = false;
            for (uint32_t rt = blockIdx.x; rt < nrt && !stop; rt += gridDim.x)
                for (uint32_t ct = 0; ct < nct && !stop; ++ct)
                    for (uint32_t kc = 0; kc < nchunks; ++kc) {
                        const uint32_t s = it % kAsStages, u = it / kAsStages;
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
                        uint8_t* st = ring + static_cast<size_t>(s) * kAsStage;
                        mbar_arrive_expect_tx(&full_bar[s], kAsStage);
                        tma_load_2d(st, &tmap_rows, &full_bar[s], static_cast<int32_t>(kc * 64),
                                    static_cast<int32_t>(rt * kAsM));
                        tma_load_2d(st + kAsA, &tmap_cent, &full_bar[s], static_cast<int32_t>(kc * 64),
                                    static_cast<int32_t>(ct * kAsN));
                        ++it;
                    }
            const uint32_t used = it < static_cast<uint32_t>(kAsStages) ? it : kAsStages;
            for (uint32_t s = 0; s < used; ++s) {
                const uint32_t uses = (it - s + kAsStages - 1) / kAsStages;
                if (!mbar_wait_bounded(&full_bar[s], (uses - 1) & 1u, kWaitBudgetCycles))
                    record_status(p.status, kStatusTimeout);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = tc::instr_desc_f16<kAsM, kAsN>();
            const uint32_t ring0 = smem_u32(ring);
            uint32_t it = 0, seq = 0;
            for (uint32_t rt = blockIdx.x; rt < nrt; rt += gridDim.x)
                for (uint32_t ct = 0; ct < nct; ++ct, ++seq) {
                    const uint32_t buf = seq & 1u, ub = seq >> 1;
                    if (ub > 0 && !*abort_flag &&
                        !mbar_wait_bounded(&tempty[buf], (ub - 1) & 1u, kWaitBudgetCycles)) {
                        *abort_flag = 1;
                        record_status(p.status, kStatusTimeout);
                    }
                    tc::fence_after_sync();
                    const uint32_t d = tmem_base + buf * kAsN;
                    for (uint32_t kc = 0; kc < nchunks; ++kc, ++it) {
                        const uint32_t s = it % kAsStages, u = it / kAsStages;
                        if (!*abort_flag && !mbar_wait_bounded(&full_bar[s], u & 1u, kWaitBudgetCycles)) {
                            *abort_flag = 1;
                            record_status(p.status, kStatusTimeout);
                        }
                        tc::fence_after_sync();
                        if (!*abort_flag) {
                            const uint32_t a_addr = ring0 + s * kAsStage, b_addr = a_addr + kAsA;
#pragma unroll
                            for (uint32_t kk = 0; kk < 4; ++kk)
                                tc::mma<false>(d, tc::smem_desc_sw128(a_addr + kk * 32),
                                               tc::smem_desc_sw128(b_addr + kk * 32), idesc, (kc | kk) != 0u ? 1u : 0u);
                        }
                        tc::commit(&empty_bar[s]);
                    }
                    tc::commit(&tfull[buf]);
                }
        }
    } else {
        const uint32_t quarter = warp & 3u;
        const uint32_t lrow = quarter * 32 + lane;
        const uint32_t taddr0 = tmem_base + ((quarter * 32u) << 16);
        const float cn = __uint_as_float(p.cmax[0]), cr = __uint_as_float(p.cmax[1]);
        uint32_t seq = 0;
        for (uint32_t rt = blockIdx.x; rt < nrt; rt += gridDim.x) {
            const uint64_t r = static_cast<uint64_t>(rt) * kAsM + lrow;
            const bool live = r < p.rows;
            // |s̃ − fl32(s)| ≤ ‖δx‖‖c‖ + ‖x̂‖‖δc‖ + accumulation + the f32 rounding of s.
            float thr = INFINITY;
            if (kMode == 1 && live) {
                const float nr = p.norm_up[r], rr = p.res_up[r];
                const float xh = nr + rr;
                const float e = (rr * cn + xh * cr + p.gamma * xh * (cn + cr) + 2.4e-7f * fmaxf(1.0f, nr * cn)) * 1.001f;
                thr = p.smax[r] - 2.0f * e;
            }
            float s1 = -INFINITY;
            uint32_t ncand = 0, first = 0;
            uint32_t* my_list = p.cand_list + (live ? r : 0) * kCandCap;
            for (uint32_t ct = 0; ct < nct; ++ct, ++seq) {
                const uint32_t buf = seq & 1u, ub = seq >> 1;
                if (!*abort_flag && !mbar_wait_bounded(&tfull[buf], ub & 1u, kWaitBudgetCycles)) {
                    *abort_flag = 1;
                    record_status(p.status, kStatusTimeout);
                }
                tc::fence_after_sync();
                const uint32_t taddr = taddr0 + buf * kAsN;
                uint32_t va[32], vb[32];
                auto process = [&](const uint32_t(&v)[32], uint32_t c) {
                    const uint32_t id0 = ct * kAsN + c * 32;
#pragma unroll
                    for (uint32_t jj = 0; jj < 32; ++jj) {
                        const float sv = __uint_as_float(v[jj]);
                        if (kMode == 0) {
                            if (sv > s1 && id0 + jj < p.nlist) s1 = sv;
                        } else if (sv >= thr && id0 + jj < p.nlist) {
                            if (ncand == 0) first = id0 + jj;
                            if (ncand < kCandCap) my_list[ncand] = id0 + jj;
                            ++ncand;
                        }
                    }
                };
                __syncwarp();
                tc::tmem_ld32(taddr, va);
                tmem_wait_ld_regs(va);
#pragma unroll
                for (uint32_t c = 0; c < kAsN / 32; c += 2) {
                    // the warp reconverges before each .sync.aligned tcgen05 instruction
                    __syncwarp();
                    tc::tmem_ld32(taddr + (c + 1) * 32, vb);
                    process(va, c);
                    __syncwarp();
                    tmem_wait_ld_regs(vb);
                    if (c + 2 < kAsN / 32) tc::tmem_ld32(taddr + (c + 2) * 32, va);
                    process(vb, c + 1);
                    if (c + 2 < kAsN / 32) {
                        __syncwarp();
                        tmem_wait_ld_regs(va);
                    }
                }
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[buf]);
            }
            if (live && !*abort_flag) {
                if (kMode == 0) {
                    p.smax[r] = s1;
                } else if (ncand == 1) {
                    p.assign[r] = first;  // every other centroid scores strictly lower, exactly
                } else if (ncand >= 2 && ncand <= kCandCap) {
                    const uint32_t pos = atomicAdd(p.cand_cnt, 1u);
                    p.cand[pos] = make_uint2(static_cast<uint32_t>(r), ncand);
                } else {  // too many candidates, or a non-finite bound (no candidate passed)
                    const uint32_t pos = atomicAdd(p.amb_cnt, 1u);
                    p.amb[pos] = static_cast<uint32_t>(r);
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem_base, kAsTmemCols);
    }
}

// Exact assignment among a row's candidates (every other centroid scores certainly lower): the
// highest dot_small, the lowest centroid index on a tie. One warp per queued row, one lane per
// candidate.
__global__ void kmeans_assign_cand_kernel(const float* __restrict__ base, uint32_t ds, uint32_t dp,
                                          const float* __restrict__ cent, const uint32_t* __restrict__ cand_list,
                                          const uint2* __restrict__ cand, const uint32_t* __restrict__ cand_cnt,
                                          uint32_t* __restrict__ assign) {
    const uint32_t n = *cand_cnt;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
        const uint2 e = cand[i];
        unsigned long long best = 0;
        if (lane < e.y) {
            const uint32_t c = cand_list[static_cast<uint64_t>(e.x) * kCandCap + lane];
            const float sc = fold_zero(dot_f64_seq(base + static_cast<uint64_t>(e.x) * ds,
                                                   cent + static_cast<uint64_t>(c) * ds, dp));
            best = make_key(sc, c);
        }
        best = warp_max_u64(best);
        if (lane == 0) assign[e.x] = key_row(best);
    }
}

// Exact assignment of the queued rows: dot_small against every centroid, strict `>` in centroid
// order (the lowest index wins a tie, src/approx.rs:466-474). One block per row.
__global__ void __launch_bounds__(256)
    kmeans_assign_exact_kernel(const float* __restrict__ base, uint32_t ds, uint32_t dp,
                               const float* __restrict__ cent_t, uint64_t ct_stride, uint32_t nlist,
                               const uint32_t* __restrict__ amb, const uint32_t* __restrict__ amb_cnt,
                               uint32_t* __restrict__ assign) {
    extern __shared__ float xs[];
    __shared__ unsigned long long wbest[8];
    const uint32_t n = *amb_cnt;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint32_t r = amb[i];
        __syncthreads();
        for (uint32_t d = threadIdx.x; d < ds; d += blockDim.x) xs[d] = base[static_cast<uint64_t>(r) * ds + d];
        __syncthreads();
        unsigned long long bk = 0;
        for (uint32_t c = threadIdx.x; c < nlist; c += blockDim.x) {
            const float s = fold_zero(dot_f64_seq_col(xs, cent_t, ct_stride, c, dp));
            const unsigned long long key = make_key(s, c);
            bk = key > bk ? key : bk;
        }
        bk = warp_max_u64(bk);
        if ((threadIdx.x & 31u) == 0) wbest[threadIdx.x >> 5] = bk;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long m = 0;
            for (uint32_t w = 0; w < blockDim.x / 32; ++w) m = wbest[w] > m ? wbest[w] : m;
            assign[r] = key_row(m);
        }
    }
}

// ------------------------------------------------------------------------------------------
// Stable counting sort of rows by cluster: per-block histograms (cluster-major), one exclusive
// scan, and a scatter that keeps row order inside each cluster (warp match + running cursors).
// ------------------------------------------------------------------------------------------
namespace {
constexpr uint32_t kSortRows = 2048;  // rows per histogram / scatter block
}

__global__ void cluster_hist_kernel(const uint32_t* __restrict__ assign, uint64_t rows, uint32_t nlist,
                                    uint32_t nblk, uint32_t* __restrict__ hist) {
    extern __shared__ uint32_t h[];
    for (uint32_t c = threadIdx.x; c < nlist; c += blockDim.x) h[c] = 0;
    __syncthreads();
    const uint64_t r0 = static_cast<uint64_t>(blockIdx.x) * kSortRows;
    const uint64_t r1 = (r0 + kSortRows) < rows ? (r0 + kSortRows) : rows;
    for (uint64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) atomicAdd(&h[assign[r]], 1u);
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < nlist; c += blockDim.x)
        hist[static_cast<uint64_t>(c) * nblk + blockIdx.x] = h[c];
}

// Exclusive scan of n u32 in place (one block; n up to a few million). out[n] = total.
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(uint32_t* __restrict__ v, uint64_t n) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x;
    const uint64_t per = (n + 1023) / 1024;
    const uint64_t b = t * per, e = (b + per) < n ? (b + per) : n;
    uint32_t s = 0;
    for (uint64_t i = b; i < e; ++i) s += v[i];
    part[t] = s;
    __syncthreads();
    for (uint32_t o = 1; o < 1024; o <<= 1) {
        const uint32_t x = t >= o ? part[t - o] : 0u;
        __syncthreads();
        part[t] += x;
        __syncthreads();
    }
    uint32_t run = part[t] - s;
    for (uint64_t i = b; i < e; ++i) {
        const uint32_t x = v[i];
        v[i] = run;
        run += x;
    }
    if (t == 1023) v[n] = part[1023];
}

__global__ void cluster_scatter_kernel(const uint32_t* __restrict__ assign, uint64_t rows, uint32_t nlist,
                                       uint32_t nblk, const uint32_t* __restrict__ off, uint32_t* __restrict__ perm) {
    extern __shared__ uint32_t cursor[];
    const uint32_t lane = threadIdx.x;  // one warp per block
    for (uint32_t c = lane; c < nlist; c += 32) cursor[c] = off[static_cast<uint64_t>(c) * nblk + blockIdx.x];
    __syncwarp();
    const uint64_t r0 = static_cast<uint64_t>(blockIdx.x) * kSortRows;
    const uint64_t r1 = (r0 + kSortRows) < rows ? (r0 + kSortRows) : rows;
    const uint32_t lt = (1u << lane) - 1u;
    for (uint64_t rb = r0; rb < r1; rb += 32) {
        const uint64_t r = rb + lane;
        const bool live = r < r1;
        const uint32_t active = __ballot_sync(0xffffffffu, live);
        if (live) {
            const uint32_t c = assign[r];
            const uint32_t peers = __match_any_sync(active, c);
            const uint32_t rank = __popc(peers & lt);
            const uint32_t base = cursor[c];
            __syncwarp(active);
            if (rank == 0) cursor[c] = base + __popc(peers);
            perm[base + rank] = static_cast<uint32_t>(r);
        }
        __syncwarp();
    }
}

// list offsets: offsets[c] = off[c·nblk] (the first block's position of cluster c); offsets[nlist] = rows.
__global__ void list_offsets_kernel(const uint32_t* __restrict__ off, uint32_t nlist, uint32_t nblk, uint64_t rows,
                                    uint32_t* __restrict__ offsets) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nlist) offsets[c] = off[static_cast<uint64_t>(c) * nblk];
    if (c == nlist) offsets[c] = static_cast<uint32_t>(rows);
}

// ------------------------------------------------------------------------------------------
// Centroid update (src/approx.rs:495-531). Sums: grid (nlist, ds/32), one warp, lane = dimension,
// the cluster's rows in row order; the loads run ahead of the (sequential) FP64 additions.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(32)
    centroid_sum_kernel(const float* __restrict__ base, uint32_t ds, const uint32_t* __restrict__ perm,
                        const uint32_t* __restrict__ offsets, double* __restrict__ sums) {
    const uint32_t c = blockIdx.x;
    const uint32_t d = blockIdx.y * 32 + threadIdx.x;
    const uint32_t b = offsets[c], e = offsets[c + 1];
    double s = 0.0;
    uint32_t i = b;
    constexpr uint32_t U = 16;
    for (; i + U <= e; i += U) {
        uint32_t r[U];
        float v[U];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) r[u] = perm[i + u];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) v[u] = base[static_cast<uint64_t>(r[u]) * ds + d];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) s = __dadd_rn(s, static_cast<double>(v[u]));
    }
    for (; i < e; ++i) s = __dadd_rn(s, static_cast<double>(base[static_cast<uint64_t>(perm[i]) * ds + d]));
    sums[static_cast<uint64_t>(c) * ds + d] = s;
}

// Mean, renormalise (norm_sq in dimension order, 1e-30 guard), empty cluster → zeros. Every
// operation is one IEEE rounding, as Rust evaluates it.
__global__ void centroid_normalize_kernel(const double* __restrict__ sums, uint32_t ds, uint32_t dp,
                                          const uint32_t* __restrict__ offsets, float* __restrict__ cent) {
    extern __shared__ double sc[];
    __shared__ double inv_norm_s;
    const uint32_t c = blockIdx.x;
    const uint32_t count = offsets[c + 1] - offsets[c];
    float* out = cent + static_cast<uint64_t>(c) * ds;
    if (count == 0) {
        for (uint32_t d = threadIdx.x; d < ds; d += blockDim.x) out[d] = 0.0f;
        return;
    }
    const double inv_count = __ddiv_rn(1.0, static_cast<double>(count));
    for (uint32_t d = threadIdx.x; d < ds; d += blockDim.x)
        sc[d] = __dmul_rn(sums[static_cast<uint64_t>(c) * ds + d], inv_count);
    __syncthreads();
    if (threadIdx.x == 0) {
        double norm_sq = 0.0;
        for (uint32_t d = 0; d < dp; ++d) norm_sq = __dadd_rn(norm_sq, __dmul_rn(sc[d], sc[d]));
        inv_norm_s = norm_sq > 1e-30 ? __ddiv_rn(1.0, __dsqrt_rn(norm_sq)) : 1.0;
    }
    __syncthreads();
    const double inv_norm = inv_norm_s;
    for (uint32_t d = threadIdx.x; d < ds; d += blockDim.x)
        out[d] = d < dp ? __double2float_rn(__dmul_rn(sc[d], inv_norm)) : 0.0f;
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------

IvfIndex::~IvfIndex() {
    cudaFree(d_reordered16);
    cudaFree(d_res16);
    cudaFree(d_centroids);
    cudaFree(d_cent_t);
    cudaFree(d_reordered);
    cudaFree(d_row_map);
    cudaFree(d_offsets);
}

IvfScratch::~IvfScratch() {
    cudaFree(d_qblock_off);
    cudaFree(d_g16);
    cudaFree(d_lane_qid);
    cudaFree(d_lane_slot);
    cudaFree(d_probes);
    cudaFree(d_pscore);
    cudaFree(d_list_cnt);
    cudaFree(d_list_fill);
    cudaFree(d_list_qoff);
    cudaFree(d_item_off);
    cudaFree(d_item_list);
    cudaFree(d_list_q);
    cudaFree(d_list_slot);
    cudaFree(d_q_slot_off);
    cudaFree(d_counters);
    cudaFree(d_ws);
    cudaFreeHost(h_probed);
}

static uint64_t isqrt_u64(uint64_t n) {
    if (n == 0) return 0;
    uint64_t x = n, y = (x + 1) / 2;
    while (y < x) {
        x = y;
        y = (x + n / x) / 2;
    }
    return x;
}

uint64_t ivf_choose_nlist(uint64_t rows) {
    if (rows < 256) return 1;
    const uint64_t s = isqrt_u64(rows);
    return s < 16 ? 16 : (s > 512 ? 512 : s);
}

uint64_t ivf_choose_nprobe(uint64_t nlist, uint64_t k, uint64_t rows) {
    const uint64_t pct = k >= 50 ? 8 : (k >= 20 ? 6 : 4);
    uint64_t nprobe = (nlist * pct + 99) / 100;
    if (nprobe < 1) nprobe = 1;
    const uint64_t nl = nlist ? nlist : 1;
    uint64_t avg = rows / nl;
    if (avg < 1) avg = 1;
    const unsigned __int128 mc = static_cast<unsigned __int128>(k) * 40;
    const uint64_t min_cand = mc > UINT64_MAX ? UINT64_MAX : static_cast<uint64_t>(mc);
    uint64_t min_nprobe = min_cand / avg + (min_cand % avg != 0);
    if (min_nprobe < 1) min_nprobe = 1;
    if (nprobe < min_nprobe) nprobe = min_nprobe;
    if (nprobe > nlist) nprobe = nlist;
    return nprobe;
}

namespace {

// Device scratch of one build, freed on every exit path.
struct BuildScratch {
    std::vector<void*> ptrs;
    ~BuildScratch() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t alloc(T*& p, size_t n) {
        p = nullptr;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(p);
        return e;
    }
};

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    Timer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

}  // namespace

// Cluster-contiguous copies of the rows for the list scans, in the order of v.d_row_map: the FP32
// rows and their BF16 copy with per-row residual bounds, whose maximum is raised into *d_eps.
// Enqueued on ix.stream.
static cudaError_t ivf_enqueue_layout(CudaIndex& ix, IvfIndex& v, unsigned int* d_eps) {
    const uint64_t rows = ix.rows, ds = ix.ds;
    const cudaStream_t s = ix.stream;
    const uint64_t kb16 = (ix.dims + 63) / 64 * 64;
    cudaError_t e;
    if ((e = cudaMalloc(&v.d_reordered, ix.rows_alloc * ds * sizeof(float))) != cudaSuccess) return e;
    cudaMemsetAsync(v.d_reordered + rows * ds, 0, (ix.rows_alloc - rows) * ds * sizeof(float), s);
    const uint32_t gb = static_cast<uint32_t>(std::min<uint64_t>((rows * 32 + 255) / 256, ix.sm_count * 16ull));
    gather_rows_kernel<<<gb, 256, 0, s>>>(ix.d_base, static_cast<uint32_t>(ds), v.d_row_map, rows, v.d_reordered);
    count_launch();
    v.kb16 = kb16;
    if ((e = cudaMalloc(&v.d_reordered16, ix.rows_alloc * kb16 * sizeof(__nv_bfloat16))) != cudaSuccess ||
        (e = cudaMalloc(&v.d_res16, rows * sizeof(float))) != cudaSuccess)
        return e;
    cudaMemsetAsync(v.d_reordered16 + rows * kb16, 0, (ix.rows_alloc - rows) * kb16 * sizeof(__nv_bfloat16), s);
    bf16_rows_kernel<<<gb, 256, 0, s>>>(v.d_reordered, static_cast<uint32_t>(ds), rows, v.d_reordered16,
                                        static_cast<uint32_t>(kb16), v.d_res16);
    count_launch();
    if ((e = launch_max_reduce(v.d_res16, rows, d_eps, s)) != cudaSuccess) return e;
    return cudaGetLastError();
}

// Once the layout has completed (v.h_offsets set): the longest list, the BF16 residual bound and
// the tensor maps of the reordered copies.
static int ivf_complete_layout(CudaIndex& ix, IvfIndex& v, unsigned int eps_bits) {
    v.max_list = 0;
    for (uint64_t c = 0; c < v.nlist; ++c) v.max_list = std::max<uint64_t>(v.max_list, v.h_offsets[c + 1] - v.h_offsets[c]);
    if (!encode_tmap_2d(&v.tmap_reordered, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, v.d_reordered, ix.ds, ix.rows_alloc,
                        ix.ds * sizeof(float), 32, 128, CU_TENSOR_MAP_SWIZZLE_128B) ||
        !encode_tmap_2d(&v.tmap_reordered16, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, v.d_reordered16, v.kb16,
                        ix.rows_alloc, v.kb16 * 2, 64, 256, CU_TENSOR_MAP_SWIZZLE_128B))
        return set_error(NNDEX_ERR_CUDA, "cuda execution error: cuTensorMapEncodeTiled failed (IVF rows)");
    std::memcpy(&v.eps16, &eps_bits, sizeof(float));
    if (ix.kb16 == 0) ix.kb16 = v.kb16;  // BF16 query copies for the tensor-core list scan
    return NNDEX_OK;
}

int ivf_build(CudaIndex& ix) {
    const uint64_t rows = ix.rows, ds = ix.ds, dp = ix.dp;
    const cudaStream_t s = ix.stream;
    uint64_t nlist = ix.opts.nlist ? ix.opts.nlist : ivf_choose_nlist(rows);
    const uint64_t iters = ix.opts.kmeans_iters ? ix.opts.kmeans_iters : 12;
    if (rows < 256 || nlist < 2) return NNDEX_OK;  // single-list index (src/approx.rs:49-59): never probed
    if (nlist > 16384)
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: nlist=%llu above the 16384 limit",
                         (unsigned long long)nlist);
    auto ivf = std::make_shared<IvfIndex>();
    IvfIndex& v = *ivf;
    v.nlist = nlist;
    v.iters = iters;
    ix.ivf_scratch.nprobe = ix.opts.nprobe;
    v.nlist_pad = (nlist + 255) / 256 * 256;
    const uint64_t kb = (ix.dims + 63) / 64 * 64;  // FP16 / BF16 row length (64-element K slabs)
    BuildScratch tmp;
    cudaError_t e = cudaSuccess;
    auto oom = [&](const char* what) { return cuda_error(e, what); };

    // ---- persistent outputs ----
    if ((e = cudaMalloc(&v.d_centroids, nlist * ds * sizeof(float))) != cudaSuccess) return oom("IVF centroids");
    if ((e = cudaMalloc(&v.d_cent_t, ds * v.nlist_pad * sizeof(float))) != cudaSuccess) return oom("IVF centroids");
    if ((e = cudaMalloc(&v.d_row_map, rows * sizeof(uint32_t))) != cudaSuccess) return oom("IVF row map");
    if ((e = cudaMalloc(&v.d_offsets, (nlist + 1) * sizeof(uint32_t))) != cudaSuccess) return oom("IVF offsets");
    cudaMemsetAsync(v.d_cent_t, 0, ds * v.nlist_pad * sizeof(float), s);

    // ---- scratch ----
    __half* b16 = nullptr;  // FP16 rows of the build (screens and the assignment GEMM)
    if ((e = tmp.alloc(b16, ix.rows_alloc * kb)) != cudaSuccess) return oom("IVF FP16 rows");
    cudaMemsetAsync(b16, 0, ix.rows_alloc * kb * sizeof(__half), s);
    float *norm_up, *res_up, *min_d, *mean_f32;
    uint32_t *chosen, *assign, *amb, *amb_cnt, *hist, *perm;
    unsigned int* cmax;
    unsigned long long* best;
    double *partial, *sums;
    KppState* kst;
    __half* c16;
    uint2* cand;
    uint32_t *cand_cnt, *cand_list;
    float* smax;
    const uint32_t nblk_sort = static_cast<uint32_t>((rows + kSortRows - 1) / kSortRows);
    if ((e = tmp.alloc(norm_up, rows)) || (e = tmp.alloc(res_up, rows)) || (e = tmp.alloc(min_d, rows)) ||
        (e = tmp.alloc(mean_f32, ds)) || (e = tmp.alloc(chosen, nlist)) || (e = tmp.alloc(assign, rows)) ||
        (e = tmp.alloc(amb, rows)) || (e = tmp.alloc(amb_cnt, 1)) ||
        (e = tmp.alloc(hist, nlist * nblk_sort + 1)) || (e = tmp.alloc(cmax, 2)) || (e = tmp.alloc(best, 1)) ||
        (e = tmp.alloc(sums, nlist * ds)) || (e = tmp.alloc(kst, 1)) || (e = tmp.alloc(c16, v.nlist_pad * kb)) ||
        (e = tmp.alloc(cand, rows)) || (e = tmp.alloc(cand_cnt, 1)) || (e = tmp.alloc(smax, rows)) ||
        (e = tmp.alloc(cand_list, rows * kCandCap)))
        return oom("IVF build scratch");
    perm = v.d_row_map;
    cudaMemsetAsync(c16, 0, v.nlist_pad * kb * sizeof(__half), s);

    Timer t_all, t_seed, t_km, t_lay;
    cudaEventRecord(t_all.a, s);
    cudaEventRecord(t_seed.a, s);
    // Row bounds (and the BF16 copy when the index keeps none).
    {
        const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>((rows + 7) / 8, ix.sm_count * 16ull));
        ivf_row_prep_kernel<<<blocks, 256, 0, s>>>(ix.d_base, static_cast<uint32_t>(ds), rows, b16,
                                                   static_cast<uint32_t>(kb), norm_up, res_up);
        count_launch();
    }
    // Medoid.
    {
        const size_t smem = 1024 + kColStages * kColStageBytes + 2 * kColStages * 8 + 16;
        auto kern = colsum_mean_kernel;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        kern<<<static_cast<unsigned>(ds / 32), 64, smem, s>>>(ix.tmap_f32, rows, mean_f32, ix.d_status);
        count_launch();
        cudaMemsetAsync(best, 0, sizeof(unsigned long long), s);
        cudaFuncSetAttribute(medoid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(ds * sizeof(float)));
        const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>((rows + 255) / 256, ix.sm_count * 8ull));
        medoid_kernel<<<blocks, 256, ds * sizeof(float), s>>>(ix.d_base, static_cast<uint32_t>(ds),
                                                               static_cast<uint32_t>(dp), rows, mean_f32, best);
        count_launch();
    }
    unsigned long long h_best = 0;
    cudaMemcpyAsync(&h_best, best, sizeof(h_best), cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "IVF medoid");
    const uint32_t medoid = 0xFFFFFFFFu - static_cast<uint32_t>(h_best & 0xFFFFFFFFu);
    cudaMemcpyAsync(chosen, &medoid, sizeof(uint32_t), cudaMemcpyHostToDevice, s);

    // k-means++ seeding.
    const float gamma = static_cast<float>(kb) * 1.2e-7f;  // K · 2^-23: FP32 accumulation of K products
    {
        KppState h{};
        h.rng = ix.opts.has_seed ? ix.opts.seed : rows * 2654435761ull + dp;
        cudaMemcpyAsync(kst, &h, sizeof(h), cudaMemcpyHostToDevice, s);
        const size_t smem = ds * sizeof(float) + kb * sizeof(__half) + kKppScanChunk * sizeof(float);
        auto kern = kpp_step_kernel;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        // One resident wave: every block streams its row range once, none waits for a second wave.
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kKppThreads, smem);
        const uint32_t blocks_target = static_cast<uint32_t>(ix.sm_count) * static_cast<uint32_t>(std::max(per_sm, 1));
        uint64_t rpb = (rows + blocks_target - 1) / blocks_target;
        rpb = (rpb + 31) / 32 * 32;
        const uint32_t nb = static_cast<uint32_t>((rows + rpb - 1) / rpb);
        if ((e = tmp.alloc(partial, nb)) != cudaSuccess) return oom("IVF seeding scratch");
        // FLT_MAX everywhere: the first step scores every row exactly.
        fill_f32_kernel<<<static_cast<unsigned>(std::min<uint64_t>((rows + 255) / 256, 65535)), 256, 0, s>>>(
            min_d, rows, FLT_MAX);
        count_launch();
        for (uint64_t c = 1; c < nlist; ++c) {
            kern<<<nb, kKppThreads, smem, s>>>(ix.d_base, b16, static_cast<uint32_t>(ds), static_cast<uint32_t>(kb),
                                               static_cast<uint32_t>(dp), rows, rpb, norm_up, res_up, gamma, min_d,
                                               partial, kst, chosen, static_cast<uint32_t>(c));
        }
        count_launch(static_cast<uint32_t>(nlist - 1));
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "IVF seeding launch");
        const uint32_t gb = static_cast<uint32_t>(std::min<uint64_t>((nlist * 32 + 255) / 256, 65535));
        gather_rows_kernel<<<gb, 256, 0, s>>>(ix.d_base, static_cast<uint32_t>(ds), chosen, nlist, v.d_centroids);
        count_launch();
    }
    cudaEventRecord(t_seed.b, s);

    // Spherical k-means.
    cudaEventRecord(t_km.a, s);
    CUtensorMap tmap_rows{}, tmap_cent{};
    if (!encode_tmap_2d(&tmap_rows, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, b16, kb, ix.rows_alloc, kb * 2, 64, 128,
                        CU_TENSOR_MAP_SWIZZLE_128B) ||
        !encode_tmap_2d(&tmap_cent, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, c16, kb, v.nlist_pad, kb * 2, 64, 256,
                        CU_TENSOR_MAP_SWIZZLE_128B))
        return set_error(NNDEX_ERR_CUDA, "cuda execution error: cuTensorMapEncodeTiled failed (IVF)");
    AssignParams ap;
    ap.rows = rows;
    ap.nlist = static_cast<uint32_t>(nlist);
    ap.nct = static_cast<uint32_t>(v.nlist_pad / kAsN);
    ap.nchunks = static_cast<uint32_t>(kb / 64);
    ap.norm_up = norm_up;
    ap.res_up = res_up;
    ap.cmax = cmax;
    ap.gamma = gamma;
    ap.assign = assign;
    ap.amb = amb;
    ap.amb_cnt = amb_cnt;
    ap.smax = smax;
    ap.cand_list = cand_list;
    ap.cand = cand;
    ap.cand_cnt = cand_cnt;
    ap.status = ix.d_status;
    cudaFuncSetAttribute(kmeans_assign_tc_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kAsSmem));
    cudaFuncSetAttribute(kmeans_assign_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kAsSmem));
    const uint32_t nrt = static_cast<uint32_t>((rows + kAsM - 1) / kAsM);
    const uint32_t as_grid = std::min<uint32_t>(nrt, static_cast<uint32_t>(ix.sm_count));
    const uint32_t cp_blocks = static_cast<uint32_t>((nlist * 32 + 255) / 256);
    cudaFuncSetAttribute(kmeans_assign_exact_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(ds * sizeof(float)));
    cudaFuncSetAttribute(cluster_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(nlist * sizeof(uint32_t)));
    cudaFuncSetAttribute(cluster_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(nlist * sizeof(uint32_t)));
    cudaFuncSetAttribute(centroid_normalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(ds * sizeof(double)));
    std::vector<uint32_t> h_amb(2 * iters, 0);
    uint32_t* d_amb_hist = nullptr;  // per iteration: rows of the full exact pass, rows decided among candidates
    if ((e = tmp.alloc(d_amb_hist, 2 * iters)) != cudaSuccess) return oom("IVF build scratch");
    for (uint64_t it = 0; it < iters; ++it) {
        cudaMemsetAsync(cmax, 0, 2 * sizeof(unsigned int), s);
        cudaMemsetAsync(amb_cnt, 0, sizeof(uint32_t), s);
        cudaMemsetAsync(cand_cnt, 0, sizeof(uint32_t), s);
        centroid_prep_kernel<<<cp_blocks, 256, 0, s>>>(v.d_centroids, static_cast<uint32_t>(ds),
                                                        static_cast<uint32_t>(nlist), c16, static_cast<uint32_t>(kb),
                                                        v.d_cent_t, v.nlist_pad, cmax);
        kmeans_assign_tc_kernel<0><<<as_grid, kAsThreads, kAsSmem, s>>>(tmap_rows, tmap_cent, ap);
        kmeans_assign_tc_kernel<1><<<as_grid, kAsThreads, kAsSmem, s>>>(tmap_rows, tmap_cent, ap);
        kmeans_assign_exact_kernel<<<ix.sm_count * 4, 256, ds * sizeof(float), s>>>(
            ix.d_base, static_cast<uint32_t>(ds), static_cast<uint32_t>(dp), v.d_cent_t, v.nlist_pad,
            static_cast<uint32_t>(nlist), amb, amb_cnt, assign);
        kmeans_assign_cand_kernel<<<ix.sm_count * 8, 256, 0, s>>>(ix.d_base, static_cast<uint32_t>(ds),
                                                                  static_cast<uint32_t>(dp), v.d_centroids, cand_list,
                                                                  cand, cand_cnt, assign);
        cudaMemcpyAsync(d_amb_hist + 2 * it, amb_cnt, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(d_amb_hist + 2 * it + 1, cand_cnt, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
        // Lists of this assignment (stable by row).
        cluster_hist_kernel<<<nblk_sort, 256, nlist * sizeof(uint32_t), s>>>(assign, rows, static_cast<uint32_t>(nlist),
                                                                             nblk_sort, hist);
        exclusive_scan_kernel<<<1, 1024, 0, s>>>(hist, nlist * nblk_sort);
        cluster_scatter_kernel<<<nblk_sort, 32, nlist * sizeof(uint32_t), s>>>(assign, rows, static_cast<uint32_t>(nlist),
                                                                               nblk_sort, hist, perm);
        list_offsets_kernel<<<static_cast<unsigned>((nlist + 1 + 255) / 256), 256, 0, s>>>(
            hist, static_cast<uint32_t>(nlist), nblk_sort, rows, v.d_offsets);
        // New centroids.
        centroid_sum_kernel<<<dim3(static_cast<unsigned>(nlist), static_cast<unsigned>(ds / 32)), 32, 0, s>>>(
            ix.d_base, static_cast<uint32_t>(ds), perm, v.d_offsets, sums);
        centroid_normalize_kernel<<<static_cast<unsigned>(nlist), 128, ds * sizeof(double), s>>>(
            sums, static_cast<uint32_t>(ds), static_cast<uint32_t>(dp), v.d_offsets, v.d_centroids);
        count_launch(11);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "IVF k-means launch");
    }
    // Dims-major copy of the final centroids for the probe.
    centroid_prep_kernel<<<cp_blocks, 256, 0, s>>>(v.d_centroids, static_cast<uint32_t>(ds), static_cast<uint32_t>(nlist),
                                                    nullptr, static_cast<uint32_t>(kb), v.d_cent_t, v.nlist_pad, nullptr);
    count_launch();
    cudaEventRecord(t_km.b, s);

    // List layout: the reordered FP32 rows and their BF16 copy.
    cudaEventRecord(t_lay.a, s);
    cudaMemsetAsync(cmax, 0, sizeof(unsigned int), s);
    if ((e = ivf_enqueue_layout(ix, v, cmax)) != cudaSuccess) return oom("IVF reordered rows");
    cudaEventRecord(t_lay.b, s);
    cudaEventRecord(t_all.b, s);

    std::vector<uint32_t> h_off(nlist + 1), h_chosen(nlist);
    KppState h_st{};
    cudaMemcpyAsync(h_off.data(), v.d_offsets, (nlist + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h_chosen.data(), chosen, nlist * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h_amb.data(), d_amb_hist, 2 * iters * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&h_st, kst, sizeof(h_st), cudaMemcpyDeviceToHost, s);
    uint32_t h_status = 0;
    unsigned int h_eps = 0;
    cudaMemcpyAsync(&h_status, ix.d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&h_eps, cmax, sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "IVF build");
    if (h_status == kStatusTimeout)
        return set_error(NNDEX_ERR_TIMEOUT, "cuda execution error: a bounded device wait timed out (IVF build)");
    if (h_status != 0) return set_error(NNDEX_ERR_CUDA, "cuda execution error: device status %u (IVF build)", h_status);

    v.h_offsets.assign(h_off.begin(), h_off.end());
    v.h_init_rows.assign(h_chosen.begin(), h_chosen.end());
    const int st = ivf_complete_layout(ix, v, h_eps);
    if (st != NNDEX_OK) return st;
    float ms = 0.0f;
    v.stats.nlist = nlist;
    v.stats.iters = iters;
    v.stats.max_list = v.max_list;
    cudaEventElapsedTime(&ms, t_all.a, t_all.b);
    v.stats.build_ms = ms;
    cudaEventElapsedTime(&ms, t_seed.a, t_seed.b);
    v.stats.seed_ms = ms;
    cudaEventElapsedTime(&ms, t_km.a, t_km.b);
    v.stats.kmeans_ms = ms;
    cudaEventElapsedTime(&ms, t_lay.a, t_lay.b);
    v.stats.layout_ms = ms;
    v.stats.seed_exact_rows = h_st.exact_rows;
    for (uint64_t i = 0; i < iters; ++i) {
        v.stats.ambiguous_rows += h_amb[2 * i];
        v.stats.candidate_rows += h_amb[2 * i + 1];
    }
    ix.ivf = std::move(ivf);
    return NNDEX_OK;
}

int ivf_restore(CudaIndex& ix, uint64_t nlist, const float* centroids, const uint64_t* offsets,
                const uint64_t* original_indices, const uint64_t* init_rows) {
    const uint64_t rows = ix.rows, ds = ix.ds, dp = ix.dp;
    const cudaStream_t s = ix.stream;
    auto bad = [](const char* why) {
        return set_error(NNDEX_ERR_INVALID_ARGUMENT, "cuda execution error: invalid IVF layout: %s", why);
    };
    if (nlist == 0) {  // the layout of an index the reference answers exactly (src/approx.rs:49-59)
        ix.ivf.reset();
        return NNDEX_OK;
    }
    if (nlist == 1) return bad("nlist must be 0 or at least 2");
    if (nlist > 16384)
        return set_error(NNDEX_ERR_UNSUPPORTED, "cuda execution error: nlist=%llu above the 16384 limit",
                         (unsigned long long)nlist);
    if (!centroids || !offsets || !original_indices) return bad("null array");
    // Lists: offsets from 0 to rows, non-decreasing; original_indices a permutation of the rows.
    if (offsets[0] != 0 || offsets[nlist] != rows) return bad("cluster offsets must run from 0 to rows");
    for (uint64_t c = 0; c < nlist; ++c)
        if (offsets[c + 1] < offsets[c]) return bad("cluster offsets must be non-decreasing");
    std::vector<uint32_t> map(rows);
    {
        std::vector<uint8_t> seen(rows, 0);
        for (uint64_t i = 0; i < rows; ++i) {
            const uint64_t r = original_indices[i];
            if (r >= rows || seen[r]) return bad("original indices must be a permutation of the rows");
            seen[r] = 1;
            map[i] = static_cast<uint32_t>(r);
        }
    }
    for (uint64_t i = 0; i < nlist * dp; ++i)
        if (!std::isfinite(centroids[i])) return bad("non-finite centroid value");
    if (init_rows)
        for (uint64_t c = 0; c < nlist; ++c)
            if (init_rows[c] >= rows) return bad("k-means++ row out of range");

    auto ivf = std::make_shared<IvfIndex>();
    IvfIndex& v = *ivf;
    v.nlist = nlist;
    v.nlist_pad = (nlist + 255) / 256 * 256;
    cudaError_t e;
    Timer t_all;
    cudaEventRecord(t_all.a, s);
    if ((e = cudaMalloc(&v.d_centroids, nlist * ds * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&v.d_cent_t, ds * v.nlist_pad * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&v.d_row_map, rows * sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaMalloc(&v.d_offsets, (nlist + 1) * sizeof(uint32_t))) != cudaSuccess)
        return cuda_error(e, "IVF layout");
    std::vector<uint32_t> off32(offsets, offsets + nlist + 1);
    unsigned int* d_eps = nullptr;
    if ((e = cudaMalloc(&d_eps, sizeof(unsigned int))) != cudaSuccess) return cuda_error(e, "IVF layout");
    BuildScratch tmp;
    tmp.ptrs.push_back(d_eps);
    cudaMemsetAsync(d_eps, 0, sizeof(unsigned int), s);
    cudaMemsetAsync(v.d_centroids, 0, nlist * ds * sizeof(float), s);
    cudaMemsetAsync(v.d_cent_t, 0, ds * v.nlist_pad * sizeof(float), s);
    if ((e = cudaMemcpy2DAsync(v.d_centroids, ds * sizeof(float), centroids, dp * sizeof(float), dp * sizeof(float),
                               nlist, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(v.d_row_map, map.data(), rows * sizeof(uint32_t), cudaMemcpyHostToDevice, s)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(v.d_offsets, off32.data(), (nlist + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s)) !=
            cudaSuccess)
        return cuda_error(e, "IVF layout upload");
    const uint64_t kb = (ix.dims + 63) / 64 * 64;
    centroid_prep_kernel<<<static_cast<unsigned>((nlist * 32 + 255) / 256), 256, 0, s>>>(
        v.d_centroids, static_cast<uint32_t>(ds), static_cast<uint32_t>(nlist), nullptr, static_cast<uint32_t>(kb),
        v.d_cent_t, v.nlist_pad, nullptr);
    count_launch();
    if ((e = ivf_enqueue_layout(ix, v, d_eps)) != cudaSuccess) return cuda_error(e, "IVF reordered rows");
    cudaEventRecord(t_all.b, s);
    unsigned int h_eps = 0;
    cudaMemcpyAsync(&h_eps, d_eps, sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
    // the host arrays above are read by the copies until the stream drains
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_error(e, "IVF layout");
    v.h_offsets.assign(offsets, offsets + nlist + 1);
    if (init_rows) v.h_init_rows.assign(init_rows, init_rows + nlist);
    else v.h_init_rows.assign(nlist, 0);
    const int st = ivf_complete_layout(ix, v, h_eps);
    if (st != NNDEX_OK) return st;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, t_all.a, t_all.b);
    v.stats.nlist = nlist;
    v.stats.max_list = v.max_list;
    v.stats.build_ms = ms;
    v.stats.layout_ms = ms;
    ix.ivf_scratch.nprobe = ix.opts.nprobe;
    ix.ivf = std::move(ivf);
    return NNDEX_OK;
}

// Σ over the stored values (row-major, rows × ds) of splitmix64(position · 2^32 + bits): a
// position-sensitive fingerprint, identical for identical stored matrices whatever the launch.
__global__ void base_checksum_kernel(const uint32_t* __restrict__ bits, uint64_t n, unsigned long long* out) {
    uint64_t acc = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t z = (i << 32) + bits[i] + 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        acc += z ^ (z >> 31);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31u) == 0) atomicAdd(out, static_cast<unsigned long long>(acc));
}

int base_checksum(CudaIndex& ix, uint64_t* out) {
    unsigned long long* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(unsigned long long));
    if (e != cudaSuccess) return cuda_error(e, "checksum");
    cudaMemsetAsync(d, 0, sizeof(unsigned long long), ix.stream);
    const uint64_t n = ix.rows * ix.ds;
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((n + 255) / 256, ix.sm_count * 8ull));
    base_checksum_kernel<<<blocks, 256, 0, ix.stream>>>(reinterpret_cast<const uint32_t*>(ix.d_base), n, d);
    count_launch();
    unsigned long long h = 0;
    cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, ix.stream);
    e = cudaStreamSynchronize(ix.stream);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_error(e, "checksum");
    *out = h;
    return NNDEX_OK;
}

}  // namespace nndex
