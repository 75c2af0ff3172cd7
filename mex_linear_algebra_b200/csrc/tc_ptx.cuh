// tc_ptx.cuh -- thin inline-PTX wrappers for the sm_100a tensor-core path:
// mbarriers, TMA tile loads, tcgen05 (TMEM alloc, UMMA issue/commit, TMEM
// loads).  Every wait is bounded (mela::kWaitLimitNs) and reports a timeout
// to the caller instead of spinning forever.
#pragma once

#include <cuda.h>
#include "mela_common.cuh"

namespace mela {
namespace ptx {

__device__ __forceinline__ u32 smem_u32(const void *p)
{
    return (u32)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(u64 *bar, u32 count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(u64 *bar, u32 bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(u64 *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(u64 *bar, u32 parity)
{
    u32 ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of `bar`.  Returns false (and sets the
// timeout bit in *err) if the phase did not complete within `limit_ns`.
__device__ __forceinline__ bool mbar_wait(u64 *bar, u32 parity, u32 *err,
                                          unsigned long long limit_ns = kWaitLimitNs)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        for (int i = 0; i < 64; ++i)
            if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) {
            if (err) atomicOr(err, kErrWaitTimeout);
            return false;
        }
    }
}

// 2-D tiled TMA load into shared memory, completion counted on `bar`.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, u64 *bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<u64>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<u64>(map)) : "memory");
}

// ---- tcgen05
__device__ __forceinline__ void tmem_alloc(u32 *slot, u32 ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(u32 taddr, u32 ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, kind::i8, one CTA.
__device__ __forceinline__ void umma_i8(u32 d_tmem, u64 a_desc, u64 b_desc, u32 idesc, u32 accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// D[tmem] (+)= (A * sfa) x (B * sfb)^T, kind::mxf4 (packed e2m1 operands,
// one UE8M0 scale per 32 values of K), one CTA.
__device__ __forceinline__ void umma_mxf4(u32 d_tmem, u64 a_desc, u64 b_desc, u32 idesc, u32 sfa_tmem,
                                          u32 sfb_tmem, u32 accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::mxf4.block_scale.block32 [%0], %1, %2, %3, [%5], [%6], p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(sfa_tmem), "r"(sfb_tmem)
        : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns from registers.
__device__ __forceinline__ void tmem_st_32x32b_x16(u32 taddr, u32 v)
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr), "r"(v)
        : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Arrive on `bar` once every previously issued UMMA of this thread completes.
__device__ __forceinline__ void umma_commit(u64 *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns: thread t gets row (lane base + t).
__device__ __forceinline__ void tmem_ld_32x32b_x32(u32 taddr, u32 (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- pairs of CTAs (a cluster of two, cta_group::2)
__device__ __forceinline__ u32 cluster_ctarank()
{
    u32 r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// Address of the same shared-memory location in CTA `rank` of the cluster.
__device__ __forceinline__ u32 mapa_shared(u32 addr, u32 rank)
{
    u32 r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
// Arrive (release at cluster scope) on an mbarrier given by its
// shared::cluster address, possibly in the other CTA of the pair.
__device__ __forceinline__ void mbar_arrive_cluster(u32 bar_cluster)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}
// Bounded wait (acquire at cluster scope) for a phase of a barrier of this
// CTA that the other CTA of the pair arrives on.
__device__ __forceinline__ bool mbar_try_wait_cluster(u64 *bar, u32 parity)
{
    u32 ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cluster(u64 *bar, u32 parity, u32 *err)
{
    if (mbar_try_wait_cluster(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        for (int i = 0; i < 64; ++i)
            if (mbar_try_wait_cluster(bar, parity)) return true;
        if (global_ns() - t0 > kWaitLimitNs) {
            if (err) atomicOr(err, kErrWaitTimeout);
            return false;
        }
    }
}
// Every thread of both CTAs arrives; returns once all have.
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.aligned;\n\tbarrier.cluster.wait.aligned;" ::: "memory");
}
// 2-D tiled TMA load into this CTA's shared memory whose completion is
// counted on an mbarrier that may live in the other CTA of the pair
// (`bar_cluster` is a shared::cluster address).  No multicast.
__device__ __forceinline__ void tma_load_2d_pair(void *dst, const CUtensorMap *map, u32 bar_cluster, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<u64>(map)), "r"(bar_cluster), "r"(x), "r"(y)
        : "memory");
}
__device__ __forceinline__ void tmem_alloc_pair(u32 *slot, u32 ncols)
{
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish_pair()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_pair(u32 taddr, u32 ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D[tmem of both CTAs] (+)= A * B^T over the pair (M = 256: each CTA holds
// 128 rows of A and 128 rows of B, the accumulator rows of its A half).
__device__ __forceinline__ void umma_i8_pair(u32 d_tmem, u64 a_desc, u64 b_desc, u32 idesc, u32 accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_mxf4_pair(u32 d_tmem, u64 a_desc, u64 b_desc, u32 idesc, u32 sfa_tmem,
                                               u32 sfb_tmem, u32 accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::mxf4.block_scale.block32 [%0], %1, %2, %3, [%5], [%6], p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(sfa_tmem), "r"(sfb_tmem)
        : "memory");
}
// Arrive on `bar` (same offset) in every CTA of `mask` once the pair's
// previously issued UMMAs complete.
__device__ __forceinline__ void umma_commit_pair(u64 *bar, unsigned short mask)
{
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"(mask)
        : "memory");
}

// Shared-memory matrix descriptor of a K-major tile written by TMA with
// 128-byte swizzle: rows of 128 bytes, 8-row core groups 1024 bytes apart.
//   bits  0-13 start address >> 4      bits 16-29 leading byte offset >> 4 (1)
//   bits 32-45 stride byte offset >> 4 bits 46-47 descriptor version (1)
//   bits 61-63 layout (2 = 128-byte swizzle)
__device__ __forceinline__ u64 desc_k_sw128(u32 saddr)
{
    return (u64)((saddr >> 4) & 0x3FFFu) | ((u64)1 << 16) | ((u64)(1024 >> 4) << 32) |
           ((u64)1 << 46) | ((u64)2 << 61);
}

// Instruction descriptor, kind::i8: unsigned 8-bit A and B (both K-major),
// signed 32-bit accumulator, M x N.
__host__ __device__ constexpr u32 idesc_i8(int M, int N)
{
    return (2u << 4)                 // D format: s32
           | (0u << 7) | (0u << 10)  // A, B: unsigned 8-bit
           | ((u32)(N >> 3) << 17) | ((u32)(M >> 4) << 24);
}

// Instruction descriptor, kind::mxf4 block-scaled: E2M1 A and B (K-major),
// UE8M0 scale factors (scale-factor byte 0 of the addressed cells), f32
// accumulator, K = 64 per instruction, M x N.
__host__ __device__ constexpr u32 idesc_mxf4(int M, int N)
{
    return (0u << 4)                 // B scale-factor byte id
           | (1u << 7) | (1u << 10)  // A, B: E2M1
           | ((u32)(N >> 3) << 17)   //
           | (1u << 23)              // scale format: UE8M0
           | ((u32)(M >> 4) << 24)   //
           | (0u << 29)              // A scale-factor byte id
           | (0u << 31);             // K = 64 (dense)
}

}  // namespace ptx
}  // namespace mela
