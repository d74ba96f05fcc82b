// Device-side helpers shared by the sm_100a kernels: mbarrier and bulk-copy
// (TMA engine) PTX wrappers with bounded waits, and the scalar arithmetic the
// reference's element kernels use (System.Numerics.Complex semantics).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tns {

// A spin on an mbarrier gives up after this long, records an error code in
// the context's device flag, and lets the kernel return. Nothing in a correct
// run waits anywhere near this long.
constexpr unsigned long long kWaitTimeoutNs = 2000000000ull;  // 2 s

enum DeviceError : int {
    kDevOk = 0,
    kDevTimeoutFull = 1,   // consumer waited for a stage that never landed
    kDevTimeoutEmpty = 2,  // producer waited for a stage that was never released
    kDevTimeoutDrain = 3,  // producer's final wait for its own copies
    kDevTimeoutSelfTest = 5,  // tns_selftest_wait: a barrier nothing arrives on
    kDevTimeoutChain = 6,     // a chained triangular solve waited for a block that never completed
};

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase of `parity` to complete, for at most kWaitTimeoutNs, and
// give up early when another warp has already recorded an error.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err, int code) {
    if (mbar_try_wait(bar, parity)) return true;
    unsigned long long start = global_timer_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 0) {
            if (*reinterpret_cast<volatile int*>(err) != 0) return false;
            if (global_timer_ns() - start > kWaitTimeoutNs) {
                atomicCAS(err, 0, code);
                return false;
            }
        }
    }
}

// The same with a caller's limit instead of kWaitTimeoutNs (the library's
// self-test of its timeout path).
__device__ __forceinline__ bool mbar_wait_bounded_ns(uint64_t* bar, uint32_t parity, int* err, int code,
                                                     unsigned long long limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    unsigned long long start = global_timer_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 0) {
            if (*reinterpret_cast<volatile int*>(err) != 0) return false;
            if (global_timer_ns() - start > limit_ns) {
                atomicCAS(err, 0, code);
                return false;
            }
        }
    }
}

// One bulk (non-tensor) copy global -> shared, completing on `bar` with a
// byte count. Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// One tiled TMA load of a 2-D box (coordinates innermost first, in elements)
// into shared memory, completing on `bar` with the box's byte count. No
// multicast. The innermost coordinate times the element size must be a
// multiple of 16 bytes; the destination is 128-byte aligned.
__device__ __forceinline__ void tma_load_2d(void* dst_smem, const void* tmap, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_addr(dst_smem)),
        "l"(tmap), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// Orders the host's (generic proxy) writes of a tensor map in global memory
// before this thread's TMA reads of it (the tensor-map proxy).
__device__ __forceinline__ void tensormap_acquire(const void* tmap) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tmap) : "memory");
}

// Per-warpgroup register reallocation (all four warps of the warpgroup execute
// it). An increase waits until registers released by a decrease are free, so
// callers must keep the warpgroups' totals within the launch's allocation.
template <int N>
__device__ __forceinline__ void reg_alloc() {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(N));
}
template <int N>
__device__ __forceinline__ void reg_dealloc() {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(N));
}

// ---------------------------------------------------------------------------
// FP64 tensor-core MMA (DMMA): D(16x8) += A(16x4) * B(4x8), fp64 throughout.
// Fragments (g = lane/4, t = lane%4): a0=(g,t) a1=(g+8,t); b0=(t,g);
// d0=(g,2t) d1=(g,2t+1) d2=(g+8,2t) d3=(g+8,2t+1).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

// ---------------------------------------------------------------------------
// Scalar arithmetic with the reference's rounding: explicit _rn intrinsics so
// that nvcc cannot contract a*b+c into one rounding where the reference
// rounds twice.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// Complex.Abs: the scaled hypot large*sqrt(1+(small/large)^2).
__device__ __forceinline__ double cabs_net(double re, double im) {
    double a = fabs(re), b = fabs(im);
    double small = a < b ? a : b;
    double large = a < b ? b : a;
    if (small == 0.0) return large;
    if (isinf(large) && !isnan(small)) return __longlong_as_double(0x7ff0000000000000ll);
    double ratio = __ddiv_rn(small, large);
    return __dmul_rn(large, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(ratio, ratio))));
}

// Lane L (0..15) of a half-warp has accumulated the 16-lane partial sums of
// .NET's ColumnOps.Dot with 256-bit Vector<double> (ColumnOps.cs:35-65):
// partial L holds the terms i = L mod 16 below the last whole 16-block, in
// index order, and partials 0..3 then take the remaining whole 4-blocks.
// Combine them as the reference does: s[l] = (a0[l] + a1[l]) + (a2[l] + a3[l]),
// total = (s0 + s1) + (s2 + s3).
__device__ __forceinline__ double netdot_combine(double acc, int L, int base) {
    const unsigned mask = 0xffffffffu;
    double a0 = __shfl_sync(mask, acc, base + (L & 3));
    double a1 = __shfl_sync(mask, acc, base + 4 + (L & 3));
    double a2 = __shfl_sync(mask, acc, base + 8 + (L & 3));
    double a3 = __shfl_sync(mask, acc, base + 12 + (L & 3));
    double s = add_rn(add_rn(a0, a1), add_rn(a2, a3));
    double s0 = __shfl_sync(mask, s, base + 0);
    double s1 = __shfl_sync(mask, s, base + 1);
    double s2 = __shfl_sync(mask, s, base + 2);
    double s3 = __shfl_sync(mask, s, base + 3);
    return add_rn(add_rn(s0, s1), add_rn(s2, s3));
}

// Math.Max / Math.Min (.NET Core): NaN propagates, +0 beats -0.
__device__ __forceinline__ double net_max(double a, double b) {
    if (a != b) {
        if (!isnan(a)) return b < a ? a : b;
        return a;
    }
    return signbit(b) ? a : b;
}

}  // namespace tns
