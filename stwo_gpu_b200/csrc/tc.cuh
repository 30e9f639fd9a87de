// Blackwell tensor-core plumbing (sm_100a): shared-memory matrix descriptors, the
// instruction descriptor of the 8-bit integer MMA, tcgen05 MMA / commit / TMEM load,
// TMEM allocation, and mbarriers whose waits give up after a time limit.
//
// Operand layout used here (K-major, no swizzle): a matrix of R rows x K bytes is stored
// as K/16 slabs of R rows x 16 bytes, slab g at g * (R * 16) bytes; inside a slab, row r
// holds bytes 16g .. 16g + 15 of its K at r * 16. Eight consecutive rows form one
// 128-byte core matrix, so the descriptor's stride between 8-row groups is 128 bytes
// and its leading offset (the next 16 bytes of K) is R * 16 bytes. One kind::i8 MMA
// consumes 32 bytes of K, i.e. two slabs.
#pragma once
#include <cstdint>

namespace stwo {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle: start address, leading byte offset (K
// direction), stride byte offset (8-row groups), each encoded >> 4; bits 46-47 hold
// the descriptor version (1 on sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of tcgen05.mma kind::i8: unsigned 8-bit A and B (format 0),
// signed 32-bit accumulator (format 2, bits 4-5), both operands K-major, N >> 3 at bits
// 17-22, M >> 4 at bits 24-28.
template <int M, int N>
__host__ __device__ constexpr uint32_t idesc_u8() {
    static_assert(M == 128, "one CTA, M = 128 rows");
    static_assert(N >= 16 && N <= 256 && N % 16 == 0, "N: a multiple of 16 up to 256");
    return (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one 128 x N x 32 step; issued by one thread.
__device__ __forceinline__ void mma_u8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// The barrier at `mbar` receives one arrival when every MMA this thread issued so far
// has completed (their shared-memory reads included).
__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's generic shared-memory writes visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation by one whole warp; the base address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit TMEM columns of this thread's lane (warp w reads lanes
// 32 (w % 4) .. 32 (w % 4) + 31); complete after tmem_wait_ld().
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

// 4-byte asynchronous copy global -> shared.
__device__ __forceinline__ void cp_async4(uint32_t dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
// The barrier at `mbar` receives one arrival (counted in its expected arrivals) when
// every asynchronous copy this thread issued so far has landed.
__device__ __forceinline__ void cp_async_arrive(uint32_t mbar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase of parity `parity` to complete, for at most limit_ns nanoseconds
// and, when abort is not null, only while *abort stays 0. Returns false on time-out or
// abort.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, const volatile uint32_t *abort,
                                          uint64_t limit_ns) {
    if (mbar_try(mbar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_try(mbar, parity)) return true;
        if (abort && *abort) return false;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

}  // namespace tc
}  // namespace stwo
