// tpsc_tc.cuh -- the pieces of the fifth-generation tensor core (tcgen05) the
// tensor slice plan uses, as inline PTX for sm_100a: tensor memory
// allocation, shared-memory matrix descriptors (no swizzle, K-major), the
// instruction descriptor of kind::tf32 with FP32 accumulation, the MMA, its
// commit to an mbarrier, bounded mbarrier waits and tensor-memory loads.
//
// Operand layout (K-major, no swizzle): a matrix of R rows (R a multiple of
// 8) and K columns is stored as K/4 column chunks of R rows x 16 bytes; chunk
// c starts at c * LBO with LBO = 16 R, and inside a chunk the 8-row core
// matrices are 128 bytes apart (SBO = 128):
//   byte(r, k) = (k / 4) * 16 R + (r / 8) * 128 + (r % 8) * 16 + (k % 4) * 4.
// One MMA consumes K = 8 (two chunks); the next K step starts 32 R bytes on.
//
// The accumulator of an M = 64 MMA occupies tensor-memory lanes
// (m % 16) + 32 (m / 16), one 32-bit column per output column: the warp
// whose rank modulo 4 is q reads rows 16 q .. 16 q + 15 with its lanes 0..15.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tpsc {
namespace {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) in a K-major operand of R rows
__host__ __device__ __forceinline__ uint32_t kmaj_off(int r, int k, int R) {
    return (uint32_t)((k >> 2) * 16 * R + (r >> 3) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// shared-memory matrix descriptor: start address, leading (K-chunk) and
// stride (8-row group) byte offsets, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::tf32: D FP32, A and B TF32, both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory made visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D (tensor memory) = A B^T (+ D when acc != 0), issued by one thread
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(acc)
        : "memory");
}
// the mbarrier completes one phase when every MMA issued so far by this thread is done
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// wait for phase `parity` of bar, bounded by max_ns of wall time: false if
// the phase did not complete in that time
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t max_ns) {
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > max_ns) return false;
    return true;
}

// 32 lanes x 16 columns: thread t receives lane (lane base + t), columns c..c+15;
// the values are valid after tmem_wait16 on the same registers
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
// wait for this thread's tensor-memory loads; the registers are tied to the
// wait so that no use of them is scheduled before it
__device__ __forceinline__ void tmem_wait16(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}
__device__ __forceinline__ void tmem_wait8(uint32_t (&r)[8]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])
                 :
                 : "memory");
}

// up to 72 columns of this warp's 32 lanes (thread t: lane base + t) into
// r[0..64) or r[0..72), then one wait; the registers are tied to the wait
__device__ __forceinline__ void tmem_ld_row72(uint32_t taddr, uint32_t (&r)[72], bool seventy_two) {
    tmem_ld16(taddr, *reinterpret_cast<uint32_t(*)[16]>(&r[0]));
    tmem_ld16(taddr + 16, *reinterpret_cast<uint32_t(*)[16]>(&r[16]));
    tmem_ld16(taddr + 32, *reinterpret_cast<uint32_t(*)[16]>(&r[32]));
    tmem_ld16(taddr + 48, *reinterpret_cast<uint32_t(*)[16]>(&r[48]));
    if (seventy_two) tmem_ld8(taddr + 64, *reinterpret_cast<uint32_t(*)[8]>(&r[64]));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 72; ++i) asm volatile("" : "+r"(r[i]));
}

// the mbarrier's current phase expects `bytes` more bytes from asynchronous copies
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// TMA: one box of a 4-D tensor map (this GPU's memory, no multicast) into
// shared memory, counted on bar
__device__ __forceinline__ void tma_load_4d(void *dst, const void *tmap, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
// bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) into shared memory, counted on bar
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// x rounded to TF32 (nearest, ties away): the high part of x, and applied to
// x - hi (exact in FP32) its remainder as the MMA reads it
__device__ __forceinline__ float tf32_hi(float x) {
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    return __uint_as_float(h);
}

}  // namespace
}  // namespace tpsc
