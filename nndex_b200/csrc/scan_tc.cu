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
constexpr int kST = 4;                // ring depth for base slabs
constexpr uint32_t kAChunk = kM * 128;
constexpr uint32_t kBChunk = kN * 128;
constexpr int kThreads = 192;         // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr uint32_t kTmemCols = 512;   // two 256-column FP32 accumulators

NNDEX_DEVICE_INLINE uint8_t* align_1024(uint8_t* p) {
    const uint32_t a = smem_u32(p);
    return p + ((1024u - (a & 1023u)) & 1023u);
}
}  // namespace

size_t tc_smem_bytes(uint32_t nchunks, uint32_t kprime) {
    size_t b = 1024;
    b += static_cast<size_t>(nchunks) * kAChunk;
    b += static_cast<size_t>(kST) * kBChunk;
    b += static_cast<size_t>(kprime) * kM * 8;
    b += 2 * kN * 4;
    b += (2 * kST + 5) * 8 + 16;
    return b;
}

template <bool kFp8>
__global__ void __launch_bounds__(kThreads, 1)
    scan_tc_kernel(const __grid_constant__ CUtensorMap tmap_q, const __grid_constant__ CUtensorMap tmap_b,
                   uint32_t nq, uint32_t nchunks, uint64_t rows, uint64_t range_rows, uint32_t kprime,
                   const float* __restrict__ row_scale, const float* __restrict__ q_scale,
                   unsigned long long* __restrict__ thr_global, uint64_t* __restrict__ ws_keys,
                   uint32_t* __restrict__ status) {
    constexpr uint32_t kElems = kFp8 ? 128 : 64;  // K elements per 128-byte slab
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = align_1024(smem_raw);
    uint8_t* a_smem = smem;
    uint8_t* b_smem = a_smem + static_cast<size_t>(nchunks) * kAChunk;
    uint64_t* heap = reinterpret_cast<uint64_t*>(b_smem + static_cast<size_t>(kST) * kBChunk);
    float* scale_s = reinterpret_cast<float*>(heap + static_cast<size_t>(kprime) * kM);
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(scale_s + 2 * kN);
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
            const uint64_t policy = l2_policy_evict_first();
            mbar_arrive_expect_tx(a_full, nchunks * kAChunk);
            for (uint32_t c = 0; c < nchunks; ++c)
                tma_load_2d(a_smem + static_cast<size_t>(c) * kAChunk, &tmap_q, a_full, static_cast<int32_t>(c * kElems),
                            static_cast<int32_t>(q0));
            uint32_t it = 0;
            bool stop = false;
            for (uint32_t t = 0; t < ntiles && !stop; ++t) {
                const int32_t y = static_cast<int32_t>(row_begin + static_cast<uint64_t>(t) * kN);
                for (uint32_t c = 0; c < nchunks; ++c) {
                    const uint32_t s = it & (kST - 1), u = it / kST;
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
                    tma_load_2d_hint(b_smem + static_cast<size_t>(s) * kBChunk, &tmap_b, &full_bar[s],
                                     static_cast<int32_t>(c * kElems), y, policy);
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
                    const uint32_t s = it & (kST - 1), u = it / kST;
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
        uint32_t n = 0;
        for (uint32_t t = 0; t < ntiles; ++t) {
            const uint32_t buf = t & 1u, ub = t >> 1;
            const uint64_t tile_row0 = row_begin + static_cast<uint64_t>(t) * kN;
            if (kFp8) {
                float* sc = scale_s + (t & 1u) * kN;
                for (uint32_t j = et; j < static_cast<uint32_t>(kN); j += 128)
                    sc[j] = (tile_row0 + j < row_end) ? row_scale[tile_row0 + j] * qs : 0.0f;
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
            const float* sc = scale_s + (t & 1u) * kN;
#pragma unroll 1
            for (uint32_t c = 0; c < kN / 32; ++c) {
                uint32_t v[32];
                __syncwarp();
                tc::tmem_ld32(tmem_base + ((quarter * 32u) << 16) + buf * kN + c * 32, v);
                tc::tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    float s = __uint_as_float(v[j]);
                    if (kFp8) s *= sc[c * 32 + j];
                    const uint64_t row = tile_row0 + c * 32 + j;
                    if (s >= thr_f && row < row_end) {
                        const uint64_t key = make_key(s, static_cast<uint32_t>(row));
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
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    rerank_kernel(const float* __restrict__ base, uint32_t ds, const float* __restrict__ queries,
                  const uint64_t* __restrict__ cand_idx, const float* __restrict__ cand_sim,
                  const uint32_t* __restrict__ cand_cnt, uint32_t kp, uint32_t k, const float* __restrict__ q_resid,
                  float eps_rows, float eps_acc, uint64_t* __restrict__ idx_out, float* __restrict__ sim_out,
                  uint32_t* __restrict__ cnt_out, uint32_t* __restrict__ cert_out) {
    extern __shared__ uint64_t keys[];
    const uint32_t q = blockIdx.x;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, nw = blockDim.x >> 5;
    const uint32_t n = cand_cnt[q] < kp ? cand_cnt[q] : kp;
    uint32_t p2 = 1;
    while (p2 < kp) p2 <<= 1;
    const float* qv = queries + static_cast<size_t>(q) * ds;
    for (uint32_t j = warp; j < p2; j += nw) {
        uint64_t key = 0;
        if (j < n) {
            const uint64_t row = cand_idx[static_cast<size_t>(q) * kp + j];
            const float* x = base + row * ds;
            float acc = 0.0f;
            for (uint32_t d = lane; d < ds; d += 32) acc = fmaf(x[d], qv[d], acc);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            key = make_key(acc, static_cast<uint32_t>(row));
        }
        if (lane == 0) keys[j] = key;
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
        // Every row outside the candidate set has an approximate score <= the k′-th candidate's,
        // so its exact score is <= tau + eps. Exact k-th above that bound => the top-k is exact.
        uint32_t ok = 1;
        if (n >= kp && kk > 0) {
            const float tau = cand_sim[static_cast<size_t>(q) * kp + kp - 1];
            const float rq = q_resid ? q_resid[q] : 0.0f;
            const float eps = eps_rows + rq * (1.0f + eps_rows) + eps_acc;
            ok = key_score(keys[kk - 1]) > tau + eps ? 1u : 0u;
        }
        cert_out[q] = ok;
    }
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
template <bool kFp8>
static cudaError_t launch_tc_impl(const TcArgs& a, cudaStream_t stream) {
    auto kern = scan_tc_kernel<kFp8>;
    const size_t smem = tc_smem_bytes(a.nchunks, a.kprime);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    dim3 grid((a.nq + kM - 1) / kM, a.nranges);
    kern<<<grid, kThreads, smem, stream>>>(*a.tmap_q, *a.tmap_b, a.nq, a.nchunks, a.rows, a.range_rows, a.kprime,
                                            a.row_scale, a.q_scale, a.thr_global, a.ws_keys, a.status);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_scan_tc(const TcArgs& a, bool fp8, cudaStream_t stream) {
    return fp8 ? launch_tc_impl<true>(a, stream) : launch_tc_impl<false>(a, stream);
}

cudaError_t launch_rerank(const RerankArgs& a, cudaStream_t stream) {
    uint32_t p2 = 1;
    while (p2 < a.kp) p2 <<= 1;
    rerank_kernel<<<a.nq, 256, p2 * sizeof(uint64_t), stream>>>(
        a.base, a.ds, a.queries, a.cand_idx, a.cand_sim, a.cand_cnt, a.kp, a.k, a.q_resid, a.eps_rows, a.eps_acc,
        a.idx_out, a.sim_out, a.cnt_out, a.cert_out);
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
