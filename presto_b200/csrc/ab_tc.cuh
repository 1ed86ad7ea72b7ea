// ab_tc.cuh -- 5th-generation tensor-core (tcgen05) primitives for sm_100a:
// tensor-memory allocation, shared-memory matrix descriptors, BF16 MMA with
// FP32 accumulation in tensor memory, commit to an mbarrier, and tensor-memory
// loads.  Field layouts follow the PTX ISA for tcgen05 (descriptor version 1).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ab {
namespace tc {

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t) __cvta_generic_to_shared(p); }

// One full warp: allocate ncols (power of two, 32..512) tensor-memory columns;
// the address is written to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)),
                 "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, no swizzle ("interleave"): 8x16 B
// core matrices; lbo = byte distance between the two K-halves of a 16-element
// K step, sbo = byte distance between groups of 8 rows.
__device__ __forceinline__ uint64_t desc_k_nosw(const void *tile, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t) ((saddr(tile) >> 4) & 0x3FFF);
    d |= (uint64_t) ((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t) ((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t) 1 << 46;                        // descriptor version (sm_100)
    // base offset 0, legacy LBO mode, layout type 0 = no swizzle
    return d;
}

// Instruction descriptor: kind::f16 with BF16 A and B (K-major), FP32 D.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N)
{
    return (1u << 4)                  // D format F32
         | (1u << 7)                  // A format BF16
         | (1u << 10)                 // B format BF16
         | ((uint32_t) (N >> 3) << 17)
         | ((uint32_t) (M >> 4) << 24);
}

// Instruction descriptor: kind::f16 with FP16 A and B (K-major), FP32 D.
__host__ __device__ constexpr uint32_t idesc_f16_f32(int M, int N)
{
    return (1u << 4)                  // D format F32; A, B format F16 (0)
         | ((uint32_t) (N >> 3) << 17)
         | ((uint32_t) (M >> 4) << 24);
}

// D[tmem] (+)= A . B^T, issued by one thread (kind::f16: A and B both BF16 or
// both FP16, as the instruction descriptor says).
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1),
          "r"(mask2), "r"(mask3)
        : "memory");
}

// Arrive on the mbarrier when every MMA issued so far by this thread is done.
__device__ __forceinline__ void commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive on bar (count 1) announcing `bytes` of asynchronous transactions.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes)
                 : "memory");
}

// Contiguous global -> shared copy by the bulk-copy engine, completing
// `bytes` of transactions on bar.  No multicast.  dst and src 16-byte
// aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(saddr(dst)), "l"(src), "r"(bytes), "r"(saddr(bar))
                 : "memory");
}

// Bounded wait on an mbarrier phase: false (and *err |= flag) if it did not
// complete within ~2^22 polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned *err, unsigned flag)
{
    for (int i = 0; i < (1 << 22); i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(saddr(bar)), "r"(parity) : "memory");
        if (done) return true;
    }
    if (err) atomicOr(err, flag);
    return false;
}

// Warp-collective: lane l gets columns [col, col+8) of tensor-memory lane
// (lane base of taddr) + l, as FP32.
__device__ __forceinline__ void ld_x8(uint32_t taddr, float (&v)[8])
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr) : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row, k) of a K-major no-swizzle tile whose rows
// hold kc elements of 2 bytes: core matrices of 8 rows x 8 elements stored
// K-contiguously (lbo = 128 B, sbo = kc/8 * 128 B).
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int kc)
{
    return (uint32_t) ((row >> 3) * (kc >> 3) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

}  // namespace tc
}  // namespace ab
