// tc.cuh — tcgen05 (5th-generation tensor core) helpers for sm_100a: TMEM allocation, shared-memory
// matrix descriptors, the instruction descriptor, MMA issue, commit, TMEM loads and fences.
//
// Descriptor formats (sm_100 UMMA):
//   shared-memory descriptor (64 bit): start address >> 4 in [0,14), leading byte offset >> 4 in
//   [16,30), stride byte offset >> 4 in [32,46), version = 1 in [46,48), base offset in [49,52),
//   layout type in [61,64) (2 = 128-byte swizzle). For a K-major operand stored as rows of 128 bytes
//   with the 128-byte swizzle, consecutive 8-row groups are 1024 bytes apart (SBO = 1024) and the
//   leading offset is unused (1). Advancing along K inside the 128-byte row moves the start address.
//   instruction descriptor (32 bit): D format in [4,6) (1 = F32), A format in [7,10), B format in
//   [10,13) (kind::f16: 0 = F16, 1 = BF16; kind::f8f6f4: 0 = E4M3), A/B major bits 15/16 (0 = K-major),
//   N >> 3 in [17,23), M >> 4 in [24,29).
#pragma once

#include "common.cuh"

namespace nndex {
namespace tc {

NNDEX_DEVICE_INLINE uint64_t smem_desc_sw128(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((smem_addr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>(1u) << 16;             // leading byte offset (unused, 16 B)
    d |= static_cast<uint64_t>(1024u >> 4) << 32;     // stride byte offset: 8 rows × 128 B
    d |= static_cast<uint64_t>(1u) << 46;             // descriptor version (sm_100)
    d |= static_cast<uint64_t>(2u) << 61;             // 128-byte swizzle
    return d;
}

// kind::f16 with BF16 inputs or kind::f8f6f4 with E4M3 inputs; F32 accumulate; both K-major.
template <bool kFp8, int M, int N>
__host__ __device__ constexpr uint32_t instr_desc() {
    return (1u << 4) | ((kFp8 ? 0u : 1u) << 7) | ((kFp8 ? 0u : 1u) << 10) |
           (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

// kind::f16 with FP16 inputs (format 0), F32 accumulate, both K-major.
template <int M, int N>
__host__ __device__ constexpr uint32_t instr_desc_f16() {
    return (1u << 4) | (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] · B[smem]ᵀ, issued by one thread.
template <bool kFp8>
NNDEX_DEVICE_INLINE void mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    const uint32_t z = 0;
    if constexpr (kFp8) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z)
            : "memory");
    }
}

// CTA-pair MMA (cta_group::2), issued by one thread of the pair's even CTA: M = 256 query rows, 128
// in each CTA's shared memory at the same offset (the descriptors' addresses), and N base rows, N/2
// in each CTA's shared memory; each CTA's TMEM receives its own 128 rows × N columns at tmem_d,
// columns [0, N/2) from the even CTA's B rows and [N/2, N) from the odd CTA's.
template <bool kFp8>
NNDEX_DEVICE_INLINE void mma_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                  uint32_t accumulate) {
    const uint32_t z = 0;
    if constexpr (kFp8) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f8f6f4 [%0], %1, %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n\t}"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n\t}"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z)
            : "memory");
    }
}

// D[tmem] (+)= A[smem] · B[smem]ᵀ with TF32 inputs (32-bit containers; the MMA uses the sign,
// exponent and top 10 mantissa bits), issued by one thread.
NNDEX_DEVICE_INLINE void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                  uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z)
        : "memory");
}

// kind::tf32, F32 accumulate, both K-major (A and B format 2 = TF32).
template <int M, int N>
__host__ __device__ constexpr uint32_t instr_desc_tf32() {
    return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

// The mbarrier at `bar` receives one arrival when every tcgen05 operation this thread issued
// before the commit has completed.
NNDEX_DEVICE_INLINE void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// CTA pair: the mbarrier at the same offset `bar` in every CTA of `cta_mask` receives one arrival
// when the pair's tcgen05 operations issued by this thread before the commit have completed.
NNDEX_DEVICE_INLINE void commit_pair(uint64_t* bar, uint16_t cta_mask) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"(cta_mask)
        : "memory");
}

NNDEX_DEVICE_INLINE void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
NNDEX_DEVICE_INLINE void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Warp-wide TMEM allocation; the column base address is written to *dst_smem.
NNDEX_DEVICE_INLINE void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
NNDEX_DEVICE_INLINE void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
NNDEX_DEVICE_INLINE void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// CTA pair: one warp of each CTA (the same warp) allocates the same columns in both CTAs' TMEM.
NNDEX_DEVICE_INLINE void tmem_alloc_pair(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
NNDEX_DEVICE_INLINE void tmem_relinquish_pair() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
NNDEX_DEVICE_INLINE void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Each thread of the warp reads 32 consecutive 32-bit columns of its own TMEM lane.
NNDEX_DEVICE_INLINE void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
}
NNDEX_DEVICE_INLINE void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Each thread of the warp reads 16 consecutive 32-bit columns of its own TMEM lane.
NNDEX_DEVICE_INLINE void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr)
        : "memory");
}
// tcgen05.wait::ld that also ties the 16 registers of the completed load.
NNDEX_DEVICE_INLINE void tmem_wait_ld16(uint32_t (&v)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                   "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),
                   "+r"(v[15])
                 :
                 : "memory");
}

}  // namespace tc
}  // namespace nndex
