// select.cuh — exact top-k selection on 64-bit result keys (see common.cuh for the key order).
//
// These replace nndex's TopKAccumulator / topk_from_scores (src/topk.rs:44-210). Instead of a
// heap per query, candidates that beat the running k-th key are appended to a shared-memory
// buffer; when it fills, an MSB-first radix select (8-bit digits) finds the exact k-th largest key
// and the buffer is compacted to exactly k keys. Because keys are unique, "keep keys >= k-th" keeps
// exactly k of them, and the result set equals the canonical top-k (similarity desc, index asc).
#pragma once

#include "common.cuh"

namespace nndex {

NNDEX_DEVICE_INLINE uint32_t lane_id() { return threadIdx.x & 31u; }

// Inclusive warp scan (sum) of a u32.
NNDEX_DEVICE_INLINE uint32_t warp_inclusive_scan(uint32_t v) {
    const uint32_t lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= static_cast<uint32_t>(o)) v += n;
    }
    return v;
}

NNDEX_DEVICE_INLINE uint64_t warp_max_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        uint64_t n = __shfl_xor_sync(0xffffffffu, v, o);
        v = n > v ? n : v;
    }
    return v;
}
NNDEX_DEVICE_INLINE uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        uint64_t n = __shfl_xor_sync(0xffffffffu, v, o);
        v = n < v ? n : v;
    }
    return v;
}

// Given a 256-bin histogram, locate the bin holding the `krem`-th largest element (1-based,
// counting from the highest bin). Executed by one full warp; returns (bin, count above, count in
// bin) in every lane.
NNDEX_DEVICE_INLINE void warp_find_bin(const uint32_t* hist, uint32_t krem, uint32_t& bin, uint32_t& above,
                                       uint32_t& in_bin) {
    const uint32_t lane = lane_id();
    uint32_t c[8];
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        c[j] = hist[255 - 8 * lane - j];
        s += c[j];
    }
    const uint32_t incl = warp_inclusive_scan(s);
    const uint32_t excl = incl - s;
    const bool mine = excl < krem && krem <= incl;
    const uint32_t ballot = __ballot_sync(0xffffffffu, mine);
    uint32_t b = 0, a = 0, n = 0;
    if (mine) {
        uint32_t run = excl;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (n == 0 && run + c[j] >= krem) {
                b = 255 - 8 * lane - j;
                a = run;
                n = c[j];
            }
            if (n == 0) run += c[j];
        }
    }
    const int src = ballot ? (__ffs(ballot) - 1) : 0;
    bin = __shfl_sync(0xffffffffu, b, src);
    above = __shfl_sync(0xffffffffu, a, src);
    in_bin = __shfl_sync(0xffffffffu, n, src);
}

// A slot from *counter (shared or global) for each lane with `take`, one atomic per warp; all 32
// lanes call it. Slots are consecutive in lane order within the warp.
NNDEX_DEVICE_INLINE uint32_t warp_append(uint32_t* counter, bool take) {
    const uint32_t ballot = __ballot_sync(0xffffffffu, take);
    if (ballot == 0u) return 0u;
    const uint32_t leader = static_cast<uint32_t>(__ffs(ballot) - 1);
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(ballot)));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + static_cast<uint32_t>(__popc(ballot & ((1u << lane_id()) - 1u)));
}

// Exact k-th largest key among buf[0..n) (requires 1 <= k <= n), by one warp. `hist` is a
// 256-entry per-warp scratch in shared memory. buf may live in shared or global memory.
NNDEX_DEVICE_INLINE uint64_t warp_radix_kth(const uint64_t* buf, uint32_t n, uint32_t k, uint32_t* hist) {
    const uint32_t lane = lane_id();
    uint64_t prefix = 0, mask = 0;
    uint32_t krem = k;
#pragma unroll 1
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (uint32_t i = lane; i < 256; i += 32) hist[i] = 0;
        __syncwarp();
        for (uint32_t i = lane; i < n; i += 32) {
            const uint64_t key = buf[i];
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 0xFFu], 1u);
        }
        __syncwarp();
        uint32_t bin, above, in_bin;
        warp_find_bin(hist, krem, bin, above, in_bin);
        __syncwarp();
        krem -= above;
        prefix |= static_cast<uint64_t>(bin) << shift;
        mask |= 0xFFull << shift;
        if (in_bin == krem) {
            // Every key in this bin is selected: the k-th is the smallest of them.
            uint64_t m = ~0ull;
            for (uint32_t i = lane; i < n; i += 32) {
                const uint64_t key = buf[i];
                if ((key & mask) == prefix && key < m) m = key;
            }
            return warp_min_u64(m);
        }
    }
    return prefix;  // all 64 bits fixed
}

// Keep keys >= thr in place (order not preserved), by one warp; returns the new count.
NNDEX_DEVICE_INLINE uint32_t warp_compact_ge(uint64_t* buf, uint32_t n, uint64_t thr) {
    const uint32_t lane = lane_id();
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t out = 0;
#pragma unroll 1
    for (uint32_t base = 0; base < n; base += 32) {
        const uint32_t i = base + lane;
        const uint64_t key = i < n ? buf[i] : 0ull;
        const bool keep = i < n && key >= thr;
        const uint32_t ballot = __ballot_sync(0xffffffffu, keep);
        __syncwarp();
        if (keep) buf[out + __popc(ballot & lt_mask)] = key;
        out += __popc(ballot);
        __syncwarp();
    }
    return out;
}

// ---- block-wide variants (used by the cross-CTA merge) -----------------------------------

struct BlockSelectScratch {
    uint32_t hist[256];
    uint32_t bin, above, in_bin;
    uint32_t count;
    unsigned long long kth;
};

// Exact k-th largest among keys[0..n) (global or shared), 1 <= k <= n. All threads of the block
// call it; warp 0 resolves bins. Keys equal to 0 take part like any other key.
NNDEX_DEVICE_INLINE uint64_t block_radix_kth(const uint64_t* keys, uint64_t n, uint32_t k, BlockSelectScratch& s) {
    uint64_t prefix = 0, mask = 0;
    uint32_t krem = k;
#pragma unroll 1
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) s.hist[i] = 0;
        __syncthreads();
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t key = keys[i];
            if ((key & mask) == prefix) atomicAdd(&s.hist[(key >> shift) & 0xFFu], 1u);
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            uint32_t bin, above, in_bin;
            warp_find_bin(s.hist, krem, bin, above, in_bin);
            if (threadIdx.x == 0) {
                s.bin = bin;
                s.above = above;
                s.in_bin = in_bin;
            }
        }
        __syncthreads();
        krem -= s.above;
        prefix |= static_cast<uint64_t>(s.bin) << shift;
        mask |= 0xFFull << shift;
        const bool done = s.in_bin == krem;
        __syncthreads();
        if (done) {
            if (threadIdx.x == 0) s.kth = ~0ull;
            __syncthreads();
            uint64_t m = ~0ull;
            for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
                const uint64_t key = keys[i];
                if ((key & mask) == prefix && key < m) m = key;
            }
            m = warp_min_u64(m);
            if ((threadIdx.x & 31) == 0) atomicMin(&s.kth, static_cast<unsigned long long>(m));
            __syncthreads();
            return s.kth;
        }
    }
    return prefix;
}

// Bitonic sort of n (power of two, <= blockDim.x * 32) keys in shared memory, descending.
NNDEX_DEVICE_INLINE void block_bitonic_sort_desc(uint64_t* a, uint32_t n) {
    for (uint32_t size = 2; size <= n; size <<= 1) {
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            __syncthreads();
            for (uint32_t t = threadIdx.x; t < n / 2; t += blockDim.x) {
                const uint32_t lo = 2 * stride * (t / stride) + (t % stride);
                const uint32_t hi = lo + stride;
                const bool desc = (lo & size) == 0;
                const uint64_t x = a[lo], y = a[hi];
                if ((x < y) == desc) {
                    a[lo] = y;
                    a[hi] = x;
                }
            }
        }
    }
    __syncthreads();
}

}  // namespace nndex
