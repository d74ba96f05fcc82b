// Fifth-generation tensor core (tcgen05) primitives for sm_100a: tensor
// memory (TMEM) allocation, the single-thread MMA issue with shared-memory
// operand descriptors, commits to mbarriers, and TMEM <-> register moves.
// Only the forms the split-precision GEMM uses: kind::i8, on one CTA
// (cta_group::1) or on a CTA pair (cta_group::2).
#pragma once

#include <cstdint>

#include "device_util.cuh"

namespace tns {

// ---- TMEM allocation (one warp, .sync.aligned) --------------------------------

// Allocates `cols` TMEM columns (a power of two >= 32) and writes the base
// address to shared memory at `dst`.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// ---- ordering between thread synchronisation and tcgen05 operations ----------
__device__ __forceinline__ void tc_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// ---- MMA ------------------------------------------------------------------------

// Shared-memory matrix descriptor of a K-major operand tile written by a TMA
// load with 128-byte swizzle: rows of 128 bytes, 8-row groups 1024 bytes
// apart (stride byte offset), descriptor version 1, layout SWIZZLE_128B. The
// tile must start on a 1024-byte boundary; the k-th 32-byte step of a row
// starts `k * 32` bytes in (the swizzle is applied by the hardware).
__device__ __forceinline__ uint64_t sw128_kmajor_desc(const void* tile, uint32_t byte_offset) {
    const uint32_t addr = smem_addr(tile) + byte_offset;
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);  // start address, 16-byte units
    d |= (uint64_t)1u << 16;                  // leading byte offset (unused with 128-byte swizzle)
    d |= (uint64_t)(1024u >> 4) << 32;        // stride byte offset: 8 rows x 128 bytes
    d |= (uint64_t)1u << 46;                  // descriptor version
    d |= (uint64_t)2u << 61;                  // layout: SWIZZLE_128B
    return d;
}

// Instruction descriptor of kind::i8: signed 8-bit A and B, both K-major,
// signed 32-bit accumulator, M x N.
__host__ __device__ constexpr uint32_t i8_instr_desc(int m, int n) {
    return (2u << 4)                    // D format: S32
           | (1u << 7)                  // A format: signed 8-bit
           | (1u << 10)                 // B format: signed 8-bit
           | ((uint32_t)(n >> 3) << 17)  // N / 8
           | ((uint32_t)(m >> 4) << 24);  // M / 16
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}

// Arrive on `bar` once every MMA this thread issued so far has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// ---- TMEM <-> registers (warp-wide: lane l reads/writes TMEM lane base+l) ----------

// 16 consecutive 32-bit columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
            taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// ---- TMA: 3-D tiled load, no multicast ---------------------------------------------
__device__ __forceinline__ void tma_load_3d(void* dst_smem, const void* tmap, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst_smem)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// ---- CTA pairs (cta_group::2): two CTAs of a cluster share one MMA ----------------
// The pair's MMA has M = 256: each CTA holds 128 rows of A and of the
// accumulator (its own TMEM) and half of B's N rows; one thread of the even
// CTA issues it. No load here multicasts: each CTA's TMA fills its own shared
// memory and reports the bytes to the even CTA's barrier.

__device__ __forceinline__ uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// Every thread of both CTAs; orders shared-memory work (barrier set-up,
// remote arrivals) before the other CTA's later accesses.
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// The shared::cluster address of this CTA's shared-memory object `p` as it
// lies in cluster CTA `rank`.
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_addr(p)), "r"(rank));
    return a;
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar_cluster) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}

__device__ __forceinline__ void tmem_alloc2(uint32_t* dst, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish2() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc2(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// D[tmem of both CTAs] (+)= A[smem of both] * B[smem of both]^T, issued by one
// thread of the even CTA.
__device__ __forceinline__ void mma_i8_pair(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                            bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}
// Arrive on the barrier at `bar`'s offset in each CTA of `cta_mask` once every
// pair MMA this thread issued so far has completed.
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar, uint16_t cta_mask) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_addr(bar)),
        "h"(cta_mask)
        : "memory");
}
// 3-D tiled load into this CTA's shared memory, completing on the barrier at
// shared::cluster address `bar_cluster` (the even CTA's).
__device__ __forceinline__ void tma_load_3d_pair(void* dst_smem, const void* tmap, int x, int y, int z,
                                                 uint32_t bar_cluster) {
    asm volatile(
        "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4}], [%5];" ::"r"(smem_addr(dst_smem)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(bar_cluster)
        : "memory");
}

}  // namespace tns
