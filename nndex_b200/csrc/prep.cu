// prep.cu — K1: validation, normalisation and padding on the device.
//
// Replaces nndex's host-side preparation (src/lib.rs:239-244, 404-411, 461-599): one warp per
// row reads the raw f32 row once (coalesced), checks finiteness, computes the squared norm,
// rejects zero-norm rows, scales by 1/sqrt(norm_sq) and writes the zero-padded row. The same
// pass emits the BF16 copy and the FP8-E4M3 copy (per-row scale) for the low-precision scans,
// and the per-row quantisation residual norms the exactness certificate uses.
//
// Arithmetic follows the reference exactly:
//   * dims >= 16 (src/lib.rs:472-473, 525-532): norm_sq = (f32) Σ (f64)x² (simsimd's FP64
//     accumulation), non-finite norm_sq → NonFiniteInput;
//   * dims < 16 and single queries (src/lib.rs:536-545, 558-569): sequential FP32 sum of x*x with
//     a per-element finite check, no fused multiply-add;
//   * norm_sq <= f32::EPSILON → ZeroNorm; inv = sqrt(norm_sq).recip() (two IEEE roundings),
//     x * inv in FP32 (src/lib.rs:547-551).
// Errors: the lowest failing row wins (the reference's row order), encoded (row << 8) | code in a
// 64-bit word reduced with atomicMin.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "common.cuh"
#include "internal.h"

namespace nndex {

constexpr uint32_t kErrNonFinite = NNDEX_ERR_NON_FINITE;
constexpr uint32_t kErrZeroNorm = NNDEX_ERR_ZERO_NORM;

NNDEX_DEVICE_INLINE void report_row_error(unsigned long long* err, uint64_t row, uint32_t code) {
    atomicMin(err, static_cast<unsigned long long>((row << 8) | code));
}

// Sequential FP32 norm (no FMA), per-element finite check, on one thread.
NNDEX_DEVICE_INLINE bool seq_norm_f32(const float* src, uint32_t dims, float& out) {
    float sq = 0.0f;
    for (uint32_t i = 0; i < dims; ++i) {
        const float v = src[i];
        if (!isfinite(v)) return false;
        sq = __fadd_rn(sq, __fmul_rn(v, v));
    }
    out = sq;
    return true;
}

// mode: 0 = normalize_rows semantics, 1 = normalize_vector semantics (sequential FP32),
//       2 = already normalised (finite check + pad only).
// Low-precision outputs are optional (nullptr to skip).
__global__ void __launch_bounds__(256) prep_rows_kernel(
    const float* __restrict__ src, uint64_t rows, uint32_t dims, uint64_t row_base,
    float* __restrict__ out, uint32_t out_stride, int mode, unsigned long long* __restrict__ err,
    __nv_bfloat16* __restrict__ out_bf16, uint32_t bf16_stride,
    uint8_t* __restrict__ out_fp8, uint32_t fp8_stride, float* __restrict__ fp8_scale,
    float* __restrict__ resid_bf16, float* __restrict__ resid_fp8) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t r = warp; r < rows; r += nwarps) {
        const float* s = src + r * dims;
        float* o = out + r * out_stride;
        const uint64_t grow = row_base + r;
        float inv = 1.0f;
        bool ok = true;
        if (mode == 2) {
            bool fin = true;
            for (uint32_t i = lane; i < dims; i += 32) fin &= isfinite(s[i]) != 0;
            fin = __all_sync(0xffffffffu, fin);
            if (!fin) {
                if (lane == 0) report_row_error(err, grow, kErrNonFinite);
                ok = false;
            }
        } else {
            float norm_sq = 0.0f;
            int code = 0;
            if (mode == 1 || dims < 16) {
                if (lane == 0) {
                    if (!seq_norm_f32(s, dims, norm_sq)) code = kErrNonFinite;
                }
                code = __shfl_sync(0xffffffffu, code, 0);
                norm_sq = __shfl_sync(0xffffffffu, norm_sq, 0);
            } else {
                double acc = 0.0;
                for (uint32_t i = lane; i < dims; i += 32) {
                    const double v = static_cast<double>(s[i]);
                    acc = fma(v, v, acc);  // exact product of two f32 values in f64
                }
#pragma unroll
                for (int o2 = 16; o2 > 0; o2 >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o2);
                norm_sq = static_cast<float>(acc);
                if (!isfinite(norm_sq)) code = kErrNonFinite;
            }
            if (code == 0 && norm_sq <= 1.1920929e-07f) code = kErrZeroNorm;
            if (code != 0) {
                if (lane == 0) report_row_error(err, grow, code);
                ok = false;
            } else {
                inv = __frcp_rn(__fsqrt_rn(norm_sq));
            }
        }
        // Write the normalised (or copied) row, zero padded to out_stride. A rejected row is
        // written as zeros (residuals 0, FP8 scale 1): its batch fails, but the scans that were
        // already queued behind this kernel then read defined values, not stale memory.
        const uint32_t live_dims = ok ? dims : 0u;
        float amax = 0.0f;
        for (uint32_t i = lane; i < out_stride; i += 32) {
            const float v = i < live_dims ? (mode == 2 ? s[i] : __fmul_rn(s[i], inv)) : 0.0f;
            o[i] = v;
            amax = fmaxf(amax, fabsf(v));
        }
        if (out_bf16 != nullptr) {
            float rb = 0.0f;
            __nv_bfloat16* ob = out_bf16 + r * bf16_stride;
            for (uint32_t i = lane; i < bf16_stride; i += 32) {
                const float v = i < live_dims ? (mode == 2 ? s[i] : __fmul_rn(s[i], inv)) : 0.0f;
                const __nv_bfloat16 b = __float2bfloat16_rn(v);
                ob[i] = b;
                const float d = v - __bfloat162float(b);
                rb = fmaf(d, d, rb);
            }
#pragma unroll
            for (int o2 = 16; o2 > 0; o2 >>= 1) rb += __shfl_xor_sync(0xffffffffu, rb, o2);
            if (lane == 0 && resid_bf16 != nullptr) resid_bf16[r] = sqrtf(rb);
        }
        if (out_fp8 != nullptr) {
#pragma unroll
            for (int o2 = 16; o2 > 0; o2 >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o2));
            // Per-row scale maps the row's max magnitude to 448 (E4M3's largest finite value).
            const float scale = amax > 0.0f ? amax / 448.0f : 1.0f;
            const float inv_scale = 1.0f / scale;
            float rf = 0.0f;
            uint8_t* of = out_fp8 + r * fp8_stride;
            for (uint32_t i = lane; i < fp8_stride; i += 32) {
                const float v = i < live_dims ? (mode == 2 ? s[i] : __fmul_rn(s[i], inv)) : 0.0f;
                const __nv_fp8_e4m3 q(v * inv_scale);
                of[i] = q.__x;
                const float d = v - static_cast<float>(q) * scale;
                rf = fmaf(d, d, rf);
            }
#pragma unroll
            for (int o2 = 16; o2 > 0; o2 >>= 1) rf += __shfl_xor_sync(0xffffffffu, rf, o2);
            if (lane == 0) {
                fp8_scale[r] = scale;
                if (resid_fp8 != nullptr) resid_fp8[r] = sqrtf(rf);
            }
        }
    }
}

void launch_prep_rows(const PrepArgs& a, cudaStream_t stream) {
    if (a.rows == 0) return;
    const uint64_t warps_needed = a.rows;
    uint64_t blocks = (warps_needed + 7) / 8;
    const uint64_t max_blocks = static_cast<uint64_t>(a.sm_count) * 16;
    if (blocks > max_blocks) blocks = max_blocks;
    prep_rows_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(
        a.src, a.rows, a.dims, a.row_base, a.out, a.out_stride, a.mode, a.err, a.out_bf16, a.bf16_stride,
        a.out_fp8, a.fp8_stride, a.fp8_scale, a.resid_bf16, a.resid_fp8);
    count_launch();
}

}  // namespace nndex
