// scan_tc.cu — K3: tensor-core (tcgen05) scan of the BF16 / FP8-E4M3 base with a fused top-k′
// filter, and K4: exact FP32 rerank of the k′ candidates with the exactness certificate.
//
// This is the large-batch path of nndex's exact search (the reference's GEMM strategies,
// src/cpu.rs:256-341): S = Q̂·X̂ᵀ on the 5th-generation tensor cores, FP32 accumulation in TMEM, and
// a per-query top-k′ of the approximate scores kept in shared memory, so scores never reach HBM.
// The k′ candidates are re-scored exactly in FP32 (K4) and the top-k returned. The result is exact
// (identical to the FP32 path's selection rule) whenever the certificate holds:
//     exact k-th score  >  approximate k′-th score + ε,
// where ε bounds |q·x − q̂·x̂| for every row (quantisation residual norms from K1, Cauchy–Schwarz,
// plus the FP32 accumulation error). Queries whose certificate fails are re-run on the FP32 path.
//
// K3 layout. One CTA = 128 queries (one TMEM lane each; the query block is the MMA's A operand,
// resident in shared memory) × one range of base rows. Warp 0 issues TMA loads of 256-row base
// tiles, one 128-byte K slab per ring stage (128 B swizzle); warp 1 issues tcgen05.mma (M = 128,
// N = 256, 4 instructions per slab) into one of two 256-column FP32 accumulators in TMEM; warps 2-5
// read the finished accumulator with tcgen05.ld (each thread one query's 256 scores), scale them
// (FP8: per-row × per-query scale) and push keys that beat the query's running k′-th key into a
// per-query min-heap in shared memory. The k′-th key of each finished range is published to a
// global per-query threshold (atomicMax), which later ranges start from. No TMA multicast.
#include <cuda_bf16.h>

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
constexpr int kThreads = 192;         // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr uint32_t kTmemCols = 512;   // two 256-column FP32 accumulators

NNDEX_DEVICE_INLINE uint8_t* align_1024(uint8_t* p) {
    const uint32_t a = smem_u32(p);
    return p + ((1024u - (a & 1023u)) & 1023u);
}
}  // namespace

size_t tc_smem_bytes(uint32_t nchunks, uint32_t kprime, uint32_t stages, bool fp8) {
    size_t b = 1024;
    b += static_cast<size_t>(nchunks) * kAChunk;
    b += static_cast<size_t>(stages) * kBChunk;
    b += static_cast<size_t>(kprime) * kM * 8;
    b += 4 * kN * 4;
    b += (2 * stages + 5) * 8 + 16;
    return b;
}

uint32_t tc_stages_for(uint32_t nchunks, uint32_t kprime, bool fp8, size_t smem_limit) {
    for (uint32_t st = 4; st >= 2; --st)
        if (tc_smem_bytes(nchunks, kprime, st, fp8) <= smem_limit) return st;
    return 0;
}

template <bool kFp8, int kST>
__global__ void __launch_bounds__(kThreads, 1)
    scan_tc_kernel(const __grid_constant__ CUtensorMap tmap_q, const __grid_constant__ CUtensorMap tmap_b,
                   uint32_t nq, uint32_t nchunks, uint64_t rows, uint64_t range_rows, uint32_t kprime,
                   const float* __restrict__ row_scale, const float* __restrict__ q_scale,
                   const float* __restrict__ row_resid, const float* __restrict__ q_resid, float eps_acc,
                   unsigned long long* __restrict__ thr_global, uint64_t* __restrict__ ws_keys,
                   uint32_t* __restrict__ status) {
    constexpr uint32_t kElems = kFp8 ? 128 : 64;  // K elements per 128-byte slab
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = align_1024(smem_raw);
    uint8_t* a_smem = smem;
    uint8_t* b_smem = a_smem + static_cast<size_t>(nchunks) * kAChunk;
    uint64_t* heap = reinterpret_cast<uint64_t*>(b_smem + static_cast<size_t>(kST) * kBChunk);
    // Per-tile row data, double-buffered by tile parity: [parity][residual bound | FP8 scale][256].
    float* rowinfo = reinterpret_cast<float*>(heap + static_cast<size_t>(kprime) * kM);
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(rowinfo + 4 * kN);
    uint64_t* empty_bar = full_bar + kST;
    uint64_t* a_full = empty_bar + kST;
    uint64_t* tfull = a_full + 1;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    volatile uint32_t* abort_flag = tmem_slot + 1;

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t q0 = blockIdx.x * kM;
    const uint32_t range = blockIdx.y, nranges = gridDim.y;
    const uint64_t row_begin = static_cast<uint64_t>(range) * range_rows;
    const uint64_t row_end = (row_begin + range_rows) < rows ? (row_begin + range_rows) : rows;
    const uint32_t ntiles = row_end > row_begin ? static_cast<uint32_t>((row_end - row_begin + kN - 1) / kN) : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kST; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(a_full, 1);
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, kTmemCols);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            tma_prefetch_desc(&tmap_q);
            tma_prefetch_desc(&tmap_b);
            // Base tiles are read by every query block of the same row range at about the same
            // time: keep them in L2 with the default policy (no evict-first hint).
            mbar_arrive_expect_tx(a_full, nchunks * kAChunk);
            for (uint32_t c = 0; c < nchunks; ++c)
                tma_load_2d(a_smem + static_cast<size_t>(c) * kAChunk, &tmap_q, a_full, static_cast<int32_t>(c * kElems),
                            static_cast<int32_t>(q0));
            uint32_t it = 0;
            bool stop = false;
            for (uint32_t t = 0; t < ntiles && !stop; ++t) {
                const int32_t y = static_cast<int32_t>(row_begin + static_cast<uint64_t>(t) * kN);
                for (uint32_t c = 0; c < nchunks; ++c) {
                    const uint32_t s = it % kST, u = it / kST;
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
                    mbar_arrive_expect_tx(&full_bar[s], kBChunk);
                    tma_load_2d(b_smem + static_cast<size_t>(s) * kBChunk, &tmap_b, &full_bar[s],
                                static_cast<int32_t>(c * kElems), y);
                    ++it;
                }
            }
            // Drain every copy this thread issued before the CTA may exit.
            if (!mbar_wait_bounded(a_full, 0, kWaitBudgetCycles)) record_status(status, kStatusTimeout);
            const uint32_t used = it < static_cast<uint32_t>(kST) ? it : kST;
            for (uint32_t s = 0; s < used; ++s) {
                const uint32_t uses = (it - s + kST - 1) / kST;
                if (!mbar_wait_bounded(&full_bar[s], (uses - 1) & 1u, kWaitBudgetCycles))
                    record_status(status, kStatusTimeout);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            constexpr uint32_t idesc = tc::instr_desc<kFp8, kM, kN>();
            if (!mbar_wait_bounded(a_full, 0, kWaitBudgetCycles)) {
                *abort_flag = 1;
                record_status(status, kStatusTimeout);
            }
            tc::fence_after_sync();
            const uint32_t a_addr0 = smem_u32(a_smem), b_addr0 = smem_u32(b_smem);
            uint32_t it = 0;
            for (uint32_t t = 0; t < ntiles; ++t) {
                const uint32_t buf = t & 1u, ub = t >> 1;
                if (ub > 0 && !*abort_flag && !mbar_wait_bounded(&tempty[buf], (ub - 1) & 1u, kWaitBudgetCycles)) {
                    *abort_flag = 1;
                    record_status(status, kStatusTimeout);
                }
                tc::fence_after_sync();
                const uint32_t d = tmem_base + buf * kN;
                for (uint32_t c = 0; c < nchunks; ++c, ++it) {
                    const uint32_t s = it % kST, u = it / kST;
                    if (!*abort_flag && !mbar_wait_bounded(&full_bar[s], u & 1u, kWaitBudgetCycles)) {
                        *abort_flag = 1;
                        record_status(status, kStatusTimeout);
                    }
                    tc::fence_after_sync();
                    if (!*abort_flag) {
                        const uint32_t a_addr = a_addr0 + c * kAChunk, b_addr = b_addr0 + s * kBChunk;
#pragma unroll
                        for (uint32_t kk = 0; kk < 4; ++kk)
                            tc::mma<kFp8>(d, tc::smem_desc_sw128(a_addr + kk * 32), tc::smem_desc_sw128(b_addr + kk * 32),
                                          idesc, (c | kk) != 0u ? 1u : 0u);
                    }
                    tc::commit(&empty_bar[s]);  // frees the slab once the MMAs above have read it
                }
                tc::commit(&tfull[buf]);  // the accumulator is complete
            }
        }
    } else {
        // ---------------- epilogue: 4 warps, one query per thread ----------------
        const uint32_t quarter = warp & 3u;
        const uint32_t lrow = quarter * 32 + lane;
        const uint32_t q = q0 + lrow;
        const bool valid_q = q < nq;
        const uint32_t et = threadIdx.x - 64;  // 0..127
        unsigned long long thr_key = valid_q ? thr_global[q] : ~0ull;
        const float qs = (kFp8 && valid_q) ? q_scale[q] : 1.0f;
        // Candidates are ranked by an upper bound of the exact score: for row r,
        //   s_r ≤ s̃_r + ‖δx_r‖(1 + ‖δq‖) + ‖δq‖ + ε_acc   (Cauchy–Schwarz on q·δx + δq·x̂, ‖q‖ = 1),
        // so every row outside the final k′ has an exact score ≤ the k′-th bound.
        const float rq = valid_q ? q_resid[q] : 0.0f;
        const float b_mul = 1.0f + rq, b_add = rq + eps_acc;
        uint32_t n = 0;
        for (uint32_t t = 0; t < ntiles; ++t) {
            const uint32_t buf = t & 1u, ub = t >> 1;
            const uint64_t tile_row0 = row_begin + static_cast<uint64_t>(t) * kN;
            {
                float* ri = rowinfo + (t & 1u) * 2 * kN;
                for (uint32_t j = et; j < static_cast<uint32_t>(kN); j += 128) {
                    const bool in = tile_row0 + j < row_end;
                    ri[j] = in ? row_resid[tile_row0 + j] : 0.0f;
                    if (kFp8) ri[kN + j] = in ? row_scale[tile_row0 + j] : 0.0f;
                }
                named_bar_sync(2, 128);
            }
            if (!*abort_flag && !mbar_wait_bounded(&tfull[buf], ub & 1u, kWaitBudgetCycles)) {
                *abort_flag = 1;
                record_status(status, kStatusTimeout);
            }
            tc::fence_after_sync();
            if ((t & 15u) == 15u && valid_q) {
                const unsigned long long g = thr_global[q];
                if (g > thr_key) thr_key = g;
            }
            float thr_f = thr_key ? key_score(thr_key) : -INFINITY;
            const float* ri = rowinfo + (t & 1u) * 2 * kN;
#pragma unroll 1
            for (uint32_t c = 0; c < kN / 32; ++c) {
                uint32_t v[32];
                __syncwarp();
                tc::tmem_ld32(tmem_base + ((quarter * 32u) << 16) + buf * kN + c * 32, v);
                tc::tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    float s = __uint_as_float(v[j]);
                    if (kFp8) s = (s * ri[kN + c * 32 + j]) * qs;
                    const float ub_s = fmaf(ri[c * 32 + j], b_mul, s + b_add);
                    const uint64_t row = tile_row0 + c * 32 + j;
                    if (ub_s >= thr_f && row < row_end) {
                        const uint64_t key = make_key(ub_s, static_cast<uint32_t>(row));
                        if (key > thr_key) {
                            // min-heap insert (index-major layout: heap[i * 128 + lrow])
                            if (n < kprime) {
                                uint32_t i = n++;
                                while (i > 0) {
                                    const uint32_t p = (i - 1) >> 1;
                                    const uint64_t hp = heap[p * kM + lrow];
                                    if (hp <= key) break;
                                    heap[i * kM + lrow] = hp;
                                    i = p;
                                }
                                heap[i * kM + lrow] = key;
                            } else {
                                uint32_t i = 0;
                                for (;;) {
                                    const uint32_t l = 2 * i + 1;
                                    if (l >= n) break;
                                    const uint32_t r = l + 1;
                                    uint64_t hm = heap[l * kM + lrow];
                                    uint32_t m = l;
                                    if (r < n) {
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
                            if (n == kprime) {
                                const uint64_t mn = heap[lrow];
                                if (mn > thr_key) thr_key = mn;
                                thr_f = key_score(thr_key);
                            }
                        }
                    }
                }
            }
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[buf]);
        }
        if (valid_q) {
            uint64_t* dst = ws_keys + (static_cast<size_t>(q) * nranges + range) * kprime;
            for (uint32_t i = 0; i < kprime; ++i) dst[i] = i < n ? heap[i * kM + lrow] : 0ull;
            if (n == kprime) atomicMax(&thr_global[q], static_cast<unsigned long long>(heap[lrow]));
        }
    }
    // ---------------- teardown: release TMEM ----------------
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem_base, kTmemCols);
    }
}

// ------------------------------------------------------------------------------------------
// K4: exact FP32 rerank of the k′ candidates + top-k + certificate. One block per query.
//
// Each candidate's FP32 dot product is computed in exactly the order of the FP32 scan
// (scan_fp32.cu): eight chains, one per 16-byte chunk position ch of each 128-byte slab, each
// accumulating its chunk's four products slab by slab with FMA; then ((c0+c1)+(c2+c3)) +
// ((c4+c5)+(c6+c7)). So a query's scores are bit-identical whichever path scored it.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    rerank_kernel(const float* __restrict__ base, uint32_t ds, const float* __restrict__ queries,
                  const uint64_t* __restrict__ cand_idx, const float* __restrict__ cand_bound,
                  const uint32_t* __restrict__ cand_cnt, uint32_t kp, uint32_t k, uint64_t* __restrict__ idx_out,
                  float* __restrict__ sim_out, uint32_t* __restrict__ cnt_out, uint32_t* __restrict__ cert_out) {
    extern __shared__ uint64_t keys[];
    const uint32_t q = blockIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ch = lane & 7u, slot = threadIdx.x >> 3;  // 8 lanes per candidate
    const uint32_t nslots = blockDim.x >> 3;
    const uint32_t n = cand_cnt[q] < kp ? cand_cnt[q] : kp;
    uint32_t p2 = 1;
    while (p2 < kp) p2 <<= 1;
    const float* qv = queries + static_cast<size_t>(q) * ds;
    const uint32_t nbox = ds / 32;
    for (uint32_t j0 = 0; j0 < p2; j0 += nslots) {
        const uint32_t j = j0 + slot;
        const bool live = j < n;
        float acc = 0.0f;
        uint64_t row = 0;
        if (live) {
            row = cand_idx[static_cast<size_t>(q) * kp + j];
            const float* x = base + row * ds + ch * 4;
            const float* y = qv + ch * 4;
            for (uint32_t bx = 0; bx < nbox; ++bx) {
                const float4 a = *reinterpret_cast<const float4*>(x + bx * 32);
                const float4 b = *reinterpret_cast<const float4*>(y + bx * 32);
                acc = fmaf(a.x, b.x, acc);
                acc = fmaf(a.y, b.y, acc);
                acc = fmaf(a.z, b.z, acc);
                acc = fmaf(a.w, b.w, acc);
            }
        }
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        acc += __shfl_xor_sync(0xffffffffu, acc, 4);
        if (ch == 0 && j < p2) keys[j] = live ? make_key(acc, static_cast<uint32_t>(row)) : 0ull;
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
        uint32_t ok = 1;
        if (n >= kp && kk > 0) ok = key_score(keys[kk - 1]) > cand_bound[static_cast<size_t>(q) * kp + kp - 1] ? 1u : 0u;
        cert_out[q] = ok;
    }
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
template <bool kFp8, int kST>
static cudaError_t launch_tc_impl(const TcArgs& a, cudaStream_t stream) {
    auto kern = scan_tc_kernel<kFp8, kST>;
    const size_t smem = tc_smem_bytes(a.nchunks, a.kprime, kST, kFp8);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    dim3 grid((a.nq + kM - 1) / kM, a.nranges);
    kern<<<grid, kThreads, smem, stream>>>(*a.tmap_q, *a.tmap_b, a.nq, a.nchunks, a.rows, a.range_rows, a.kprime,
                                            a.row_scale, a.q_scale, a.row_resid, a.q_resid, a.eps_acc, a.thr_global,
                                            a.ws_keys, a.status);
    count_launch();
    return cudaGetLastError();
}

template <bool kFp8>
static cudaError_t launch_tc_stages(const TcArgs& a, cudaStream_t stream) {
    switch (a.stages) {
        case 4: return launch_tc_impl<kFp8, 4>(a, stream);
        case 3: return launch_tc_impl<kFp8, 3>(a, stream);
        case 2: return launch_tc_impl<kFp8, 2>(a, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_scan_tc(const TcArgs& a, bool fp8, cudaStream_t stream) {
    return fp8 ? launch_tc_stages<true>(a, stream) : launch_tc_stages<false>(a, stream);
}

cudaError_t launch_rerank(const RerankArgs& a, cudaStream_t stream) {
    uint32_t p2 = 1;
    while (p2 < a.kp) p2 <<= 1;
    rerank_kernel<<<a.nq, 256, p2 * sizeof(uint64_t), stream>>>(a.base, a.ds, a.queries, a.cand_idx, a.cand_sim,
                                                               a.cand_cnt, a.kp, a.k, a.idx_out, a.sim_out,
                                                               a.cnt_out, a.cert_out);
    count_launch();
    return cudaGetLastError();
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
