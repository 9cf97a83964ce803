// nan_tcgen05.cuh -- thin inline-PTX layer over the sm_100a tensor-core
// instructions used by the learned radiance cache: TMEM allocation, BF16
// tcgen05.mma with operands in shared memory, commit to an mbarrier,
// bounded mbarrier waits and TMEM loads.
//
// Shared-memory operand layout ("interleaved", no swizzle). A bf16 tile of
// R rows x C columns (C a multiple of 8) stores element (r, c) at byte
//     (r / 8) * (C * 16) + (c / 8) * 128 + (r % 8) * 16 + (c % 8) * 2,
// i.e. 8x8 core matrices of 128 contiguous bytes, the C/8 core matrices of
// an 8-row group side by side. One tile serves as
//   K-major operand  (rows = M or N, columns = K): LBO = 128,    SBO = C * 16;
//   MN-major operand (columns = M or N, rows = K): LBO = C * 16, SBO = 128.
// A K step of 16 advances the start address by 256 bytes (K-major) or by
// 2 * C * 16 bytes (MN-major).
#pragma once

#include <cstdint>

namespace nbd {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, c) in an interleaved tile of `cols` columns.
__host__ __device__ constexpr uint32_t tile_offset(uint32_t r, uint32_t c, uint32_t cols) {
    return (r >> 3) * (cols * 16u) + (c >> 3) * 128u + (r & 7u) * 16u + (c & 7u) * 2u;
}

// Shared-memory matrix descriptor, no swizzle (layout type 0), sm_100
// descriptor version 1 at bits 46-47.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    return d;
}

// Instruction descriptor of kind::f16 with BF16 A/B and FP32 D: D format at
// bits 4-5, A and B formats at 7-9 and 10-12, A/B major at 15/16 (1 = MN),
// N >> 3 at 17-22, M >> 4 at 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t m, uint32_t n, uint32_t a_mn, uint32_t b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn << 15) | (b_mn << 16) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive once on `bar` when every MMA this thread issued so far completes.
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" : : : "memory");
}

// Bounded wait for the phase with parity `parity` to complete. Returns false
// after `limit` polls (the caller records an error and leaves its loop).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = smem_addr(bar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" : : : "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" : : : "memory");
}
// Generic-proxy shared-memory writes become visible to the tensor core.
__device__ __forceinline__ void fence_smem_to_async() {
    asm volatile("fence.proxy.async.shared::cta;" : : : "memory");
}

// Whole-warp TMEM allocation; the base address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_addr(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" : : : "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(base), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit columns of this thread's TMEM lane (lane = the
// warp's quarter of the 128 lanes + lane id), waited for.
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    // the registers are tied to the wait so no use of them moves above it
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace nbd
