// common.cuh — device helpers shared by the nndex B200 kernels (sm_100a).
//
// Result keys. A (similarity, row) pair is packed into one 64-bit key whose unsigned order is
// nndex's result order: similarity descending by f32::total_cmp, then row index ascending
// (src/topk.rs:25-31, 143-148). High word: the f32 bits mapped to an order-preserving u32
// (sign-magnitude → biased); low word: 0xFFFFFFFF - row. A larger key is a better result and
// keys of distinct rows never tie, so top-k selection is a selection of the k largest keys.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#ifndef NNDEX_DEVICE_INLINE
#define NNDEX_DEVICE_INLINE __device__ __forceinline__
#endif

namespace nndex {

// Device status word values (kernel → host). 0 = clean.
enum DeviceStatus : uint32_t {
    kStatusOk = 0,
    kStatusTimeout = 1,        // a bounded mbarrier / flag wait ran out
    kStatusOverflow = 2,       // a candidate buffer would have overflowed (never expected)
    kStatusBadLaunch = 3,      // launch parameters violated a kernel precondition
};

// ---- keys ------------------------------------------------------------------------------

NNDEX_DEVICE_INLINE uint32_t float_to_ordered(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
NNDEX_DEVICE_INLINE float ordered_to_float(uint32_t u) {
    uint32_t b = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
    return __uint_as_float(b);
}
NNDEX_DEVICE_INLINE uint64_t make_key(float score, uint32_t row) {
    return (static_cast<uint64_t>(float_to_ordered(score)) << 32) | static_cast<uint64_t>(0xFFFFFFFFu - row);
}
NNDEX_DEVICE_INLINE float key_score(uint64_t key) { return ordered_to_float(static_cast<uint32_t>(key >> 32)); }
NNDEX_DEVICE_INLINE uint32_t key_row(uint64_t key) { return 0xFFFFFFFFu - static_cast<uint32_t>(key & 0xFFFFFFFFu); }

// ---- shared-memory addresses -----------------------------------------------------------

NNDEX_DEVICE_INLINE uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarrier ----------------------------------------------------------------------------

NNDEX_DEVICE_INLINE void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
NNDEX_DEVICE_INLINE void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
NNDEX_DEVICE_INLINE void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
NNDEX_DEVICE_INLINE void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
NNDEX_DEVICE_INLINE void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
NNDEX_DEVICE_INLINE bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// try_wait that may suspend the thread for up to `ns` nanoseconds while the phase is incomplete
// (a producer that mostly waits then takes no issue slots from the warps it shares a scheduler with).
NNDEX_DEVICE_INLINE bool mbar_try_wait_suspend(uint64_t* bar, uint32_t parity, uint32_t ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}

// Bounded wait with suspension: as mbar_wait_bounded, each try suspending for up to `ns`.
NNDEX_DEVICE_INLINE bool mbar_wait_bounded_suspend(uint64_t* bar, uint32_t parity, long long budget, uint32_t ns) {
    if (mbar_try_wait_suspend(bar, parity, ns)) return true;
    long long start = clock64();
    while (!mbar_try_wait_suspend(bar, parity, ns)) {
        if (clock64() - start > budget) return false;
    }
    return true;
}

// Bounded wait: spins on try_wait until the phase with `parity` completes or `budget` clock
// cycles pass. Returns false on timeout (the caller records kStatusTimeout and drains).
NNDEX_DEVICE_INLINE bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long budget) {
    if (mbar_try_wait(bar, parity)) return true;
    long long start = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - start > budget) return false;
    }
    return true;
}

// ---- thread-block clusters -------------------------------------------------------------

NNDEX_DEVICE_INLINE uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// The shared::cluster address of the variable at `p` in the cluster's CTA `rank`.
NNDEX_DEVICE_INLINE uint32_t cluster_map(const void* p, uint32_t rank) {
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
    return a;
}
// One arrival on an mbarrier of any CTA of the cluster (release at cluster scope).
NNDEX_DEVICE_INLINE void mbar_arrive_cluster(uint32_t bar_cluster) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}
// Every thread of every CTA of the cluster (all of them execute it).
NNDEX_DEVICE_INLINE void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// ≈1 s at B200 clocks: far above any legitimate wait in these kernels.
constexpr long long kWaitBudgetCycles = 2000000000ll;

// ---- TMA (no multicast anywhere in this library) -----------------------------------------

NNDEX_DEVICE_INLINE void tma_prefetch_desc(const void* tmap) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// 2-D tiled load of one box into shared memory, completing on `bar` (complete_tx::bytes).
// x is the innermost coordinate (elements) and must be a multiple of 16 bytes / element size.
NNDEX_DEVICE_INLINE void tma_load_2d(void* dst, const void* tmap, uint64_t* bar, int32_t x, int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// CTA pair (cta_group::2): the box lands in this CTA's shared memory at `dst` and its bytes complete
// on the mbarrier at shared::cluster address `bar_cluster` (the pair's even CTA's barrier). No
// multicast: each CTA loads its own box.
NNDEX_DEVICE_INLINE void tma_load_2d_pair(void* dst, const void* tmap, uint32_t bar_cluster, int32_t x, int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(bar_cluster), "r"(x), "r"(y)
        : "memory");
}

// Same, with an L2 cache policy operand (e.g. evict-first for a single streaming pass).
NNDEX_DEVICE_INLINE void tma_load_2d_hint(void* dst, const void* tmap, uint64_t* bar, int32_t x, int32_t y,
                                          uint64_t policy) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%3, %4}], [%2], %5;" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y), "l"(policy)
        : "memory");
}

NNDEX_DEVICE_INLINE uint64_t l2_policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
NNDEX_DEVICE_INLINE uint64_t l2_policy_evict_normal() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}
NNDEX_DEVICE_INLINE uint64_t l2_policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Shared-memory vector load by 32-bit shared address. Volatile: it keeps program order with the
// (volatile) mbarrier waits and barriers, so it never reads a slab before the wait that publishes it.
NNDEX_DEVICE_INLINE float4 lds128(uint32_t addr) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
    return v;
}

// Named barrier over a subset of warps (id 1..15; id 0 is __syncthreads).
NNDEX_DEVICE_INLINE void named_bar_sync(uint32_t id, uint32_t threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Record the first non-zero status (first writer wins).
NNDEX_DEVICE_INLINE void record_status(uint32_t* status, uint32_t code) {
    if (status) atomicCAS(status, 0u, code);
}

}  // namespace nndex
