// LU with partial pivoting and the triangular solves, on the GPU, for one
// matrix or a batch of independent matrices advanced in lockstep.
//
// Right-looking blocked getrf as the reference runs it (src/Tensile.Kernels/Lu.cs:230-309
// for real, src/Tensile/BlockedLu.cs:45-101 for complex): per block of nb
// columns
//   1. panel factorization (one CTA per matrix; pivot = first index of the
//      largest |a|, or |Re|+|Im| for complex; reciprocal multiply unless
//      |pivot| < SafeMin; rank-1 updates y + (-m)*x with two roundings),
//   2. the panel's row interchanges applied to the columns either side,
//   3. U12 := L11^-1 A12 (one warp per column, the reference's update order),
//   4. A22 := A22 - A21*U12 on the DMMA GEMM (bit-identical to the
//      reference's product, gemm.cu).
// Every step's arithmetic is the reference's, so the factors and pivots match
// the reference bit for bit. In a batch, step k of every matrix runs in one
// launch per phase (a grouped GEMM for the trailing updates).
//
// Solves: forward and backward substitution in the reference's order, blocked
// into 32-row diagonal solves and register-tiled updates that continue each
// element's chain of roundings in the reference's order, so A^-1 B -- the Pade
// solve included -- matches the reference bit for bit. The adjoint solves,
// whose reference order is an inner product per row, run left-looking: ColumnOps.Dot's
// vector order for real factors, sequential sums for complex ones (the forward
// half of the complex adjoint, whose sums run in ascending k, right-looking
// over the conjugate transpose), so they match bit for bit too.

#include "batch.cuh"
#include "device_util.cuh"
#include "tns_internal.h"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <type_traits>
#include <vector>

namespace tns {

namespace {

constexpr double kSafeMin = 2.2250738585072014e-308;

struct Z {
    double re, im;
};
__device__ __forceinline__ Z zload(const double* p) {
    double2 v = *reinterpret_cast<const double2*>(p);
    return {v.x, v.y};
}
__device__ __forceinline__ void zstore(double* p, Z z) { *reinterpret_cast<double2*>(p) = make_double2(z.re, z.im); }
__device__ __forceinline__ Z zmul(Z a, Z b) {
    return {sub_rn(mul_rn(a.re, b.re), mul_rn(a.im, b.im)), add_rn(mul_rn(a.im, b.re), mul_rn(a.re, b.im))};
}
__device__ __forceinline__ Z zadd(Z a, Z b) { return {add_rn(a.re, b.re), add_rn(a.im, b.im)}; }
// Smith's division, as System.Numerics.Complex divides.
__device__ __forceinline__ Z zdiv(Z l, Z r) {
    double a = l.re, b = l.im, c = r.re, d = r.im;
    if (fabs(d) < fabs(c)) {
        double doc = __ddiv_rn(d, c);
        double den = add_rn(c, mul_rn(d, doc));
        return {__ddiv_rn(add_rn(a, mul_rn(b, doc)), den), __ddiv_rn(sub_rn(b, mul_rn(a, doc)), den)};
    }
    double cod = __ddiv_rn(c, d);
    double den = add_rn(d, mul_rn(c, cod));
    return {__ddiv_rn(add_rn(b, mul_rn(a, cod)), den), __ddiv_rn(add_rn(-a, mul_rn(b, cod)), den)};
}

// ---------------------------------------------------------------------------
// Panel factorization: rows [r0, m) x columns [r0, r0 + w) of a (ld elements),
// one CTA per item. Pivots land as global 0-based rows in piv[r0 + j].
// ---------------------------------------------------------------------------
struct PanelFactorDesc {
    double* a;
    int ld, m, r0, w;
    int* piv;
    int* singular;
};

template <bool CPLX>
__global__ void __launch_bounds__(512) panel_kernel(const __grid_constant__ Batch<PanelFactorDesc> b) {
    const PanelFactorDesc& d = batch_item(b, blockIdx.x);
    constexpr int ES = CPLX ? 2 : 1;
    __shared__ double s_val[32];
    __shared__ int s_idx[32];
    __shared__ int s_p;
    __shared__ double s_prow[2 * 64];
    const int tid = threadIdx.x;
    const int nthreads = blockDim.x;
    const int ld = d.ld, w = d.w, r0 = d.r0;
    const int M = d.m - r0;  // rows in the panel
    const int limit = min(M, w);
    double* P = d.a + ((size_t)r0 * ld + r0) * ES;  // panel origin

    for (int j = 0; j < limit; ++j) {
        // a. first index of the largest pivot measure in column j, rows j..M-1
        double best = -1.0;
        int bidx = INT_MAX;
        for (int i = j + tid; i < M; i += nthreads) {
            const double* e = P + ((size_t)j * ld + i) * ES;
            double v = CPLX ? add_rn(fabs(e[0]), fabs(e[1])) : fabs(e[0]);
            if (v > best || (v == best && i < bidx)) {
                best = v;
                bidx = i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
            if (ov > best || (ov == best && oi < bidx)) {
                best = ov;
                bidx = oi;
            }
        }
        if ((tid & 31) == 0) {
            s_val[tid >> 5] = best;
            s_idx[tid >> 5] = bidx;
        }
        __syncthreads();
        if (tid == 0) {
            double bv = s_val[0];
            int bi = s_idx[0];
            for (int q = 1; q < (nthreads >> 5); ++q)
                if (s_val[q] > bv || (s_val[q] == bv && s_idx[q] < bi)) {
                    bv = s_val[q];
                    bi = s_idx[q];
                }
            // A column of NaNs (no comparison succeeds) keeps the diagonal.
            if (bi == INT_MAX) bi = j;
            s_p = bi;
            d.piv[r0 + j] = r0 + bi;
        }
        __syncthreads();
        const int p = s_p;
        // b. swap rows j and p across the panel's w columns
        if (p != j) {
            for (int c = tid; c < w; c += nthreads) {
                double* x = P + ((size_t)c * ld + j) * ES;
                double* y = P + ((size_t)c * ld + p) * ES;
                for (int q = 0; q < ES; ++q) {
                    double tmp = x[q];
                    x[q] = y[q];
                    y[q] = tmp;
                }
            }
        }
        __syncthreads();
        // c. pivot row (columns j..w-1) into shared memory
        for (int c = j + tid; c < w; c += nthreads) {
            const double* e = P + ((size_t)c * ld + j) * ES;
            s_prow[2 * c] = e[0];
            s_prow[2 * c + 1] = CPLX ? e[1] : 0.0;
        }
        __syncthreads();
        // d. scale column j below the diagonal, rank-1 update of columns j+1..w-1
        if (!CPLX) {
            double value = s_prow[2 * j];
            if (value == 0.0) {
                if (tid == 0) atomicMin(d.singular, r0 + j);
            }
            bool recip = fabs(value) >= kSafeMin;
            double r = __ddiv_rn(1.0, value);
            for (int i = j + 1 + tid; i < M; i += nthreads) {
                double* col = P + (size_t)j * ld + i;
                double l = *col;
                if (value != 0.0) {
                    l = recip ? mul_rn(l, r) : __ddiv_rn(l, value);
                    *col = l;
                }
                for (int c = j + 1; c < w; ++c) {
                    double mult = s_prow[2 * c];
                    if (mult != 0.0) {
                        double* t = P + (size_t)c * ld + i;
                        *t = add_rn(*t, mul_rn(-mult, l));
                    }
                }
            }
        } else {
            Z value{s_prow[2 * j], s_prow[2 * j + 1]};
            bool zero = value.re == 0.0 && value.im == 0.0;
            if (zero && tid == 0) atomicMin(d.singular, r0 + j);
            bool recip = cabs_net(value.re, value.im) >= kSafeMin;
            Z r = zdiv(Z{1.0, 0.0}, value);
            for (int i = j + 1 + tid; i < M; i += nthreads) {
                double* col = P + ((size_t)j * ld + i) * 2;
                Z l = zload(col);
                if (!zero) {
                    l = recip ? zmul(l, r) : zdiv(l, value);
                    zstore(col, l);
                }
                for (int c = j + 1; c < w; ++c) {
                    Z mult{s_prow[2 * c], s_prow[2 * c + 1]};
                    if (mult.re == 0.0 && mult.im == 0.0) continue;
                    Z scale{-mult.re, -mult.im};
                    double* t = P + ((size_t)c * ld + i) * 2;
                    zstore(t, zadd(zload(t), zmul(scale, l)));
                }
            }
        }
        __syncthreads();
    }
}

// The same factorization with the panel's columns taken kPanelSub at a
// time: the sub-panel (its rows j0.. of kPanelSub columns) is factored in
// shared memory column by column exactly as above, then its updates reach
// the panel's later columns in one pass: their kPanelSub pivot rows first
// (each element's updates by the earlier pivot rows of the sub-panel, in
// order), then every row below, updates in order. Every element receives the
// same operations in the same order as in panel_kernel (the updates are
// regrouped per element, never reordered; row interchanges act on the later
// columns' values as they stand, which carry the same rows), so factors and
// pivots are identical; the later columns are read and written once per
// sub-panel instead of once per column. Shared memory: kPanelSub columns of
// smem_rows rows and the sub-panel's pivot rows over up to 64 columns.
constexpr int kPanelSub = 8;
constexpr int kPanelMaxWidth = 64;

template <bool CPLX>
__global__ void __launch_bounds__(512) panel_blocked_kernel(const __grid_constant__ Batch<PanelFactorDesc> b,
                                                           int smem_rows) {
    const PanelFactorDesc& d = batch_item(b, blockIdx.x);
    constexpr int ES = CPLX ? 2 : 1;
    extern __shared__ __align__(16) double pb_smem[];
    double* S = pb_smem;                                     // S[(cc * smem_rows + i) * ES]: column j0 + cc, row j0 + i
    double* U = pb_smem + (size_t)kPanelSub * smem_rows * ES;  // U[(k * kPanelMaxWidth + c) * ES]
    __shared__ double s_val[16];
    __shared__ int s_idx[16];
    const int tid = threadIdx.x, nthreads = blockDim.x, warps = nthreads >> 5;
    const int ld = d.ld, w = d.w, r0 = d.r0;
    const int M = d.m - r0;
    const int limit = min(M, w);
    double* P = d.a + ((size_t)r0 * ld + r0) * ES;  // panel origin
    auto ldz = [](const double* e) { return Z{e[0], CPLX ? e[1] : 0.0}; };
    auto stz = [](double* e, Z v) {
        e[0] = v.re;
        if (CPLX) e[1] = v.im;
    };
    // t + (-mult) l with the panel kernel's roundings
    auto upd = [](Z t, Z mult, Z l) {
        if (!CPLX) return Z{add_rn(t.re, mul_rn(-mult.re, l.re)), 0.0};
        return zadd(t, zmul(Z{-mult.re, -mult.im}, l));
    };
    auto nonzero = [](Z v) { return CPLX ? !(v.re == 0.0 && v.im == 0.0) : v.re != 0.0; };

    for (int j0 = 0; j0 < limit; j0 += kPanelSub) {
        const int sb = min(kPanelSub, limit - j0), Mr = M - j0;
        for (int e = tid; e < Mr * sb; e += nthreads) {
            const int i = e % Mr, cc = e / Mr;
            stz(S + ((size_t)cc * smem_rows + i) * ES, ldz(P + ((size_t)(j0 + cc) * ld + j0 + i) * ES));
        }
        __syncthreads();
        for (int jj = 0; jj < sb; ++jj) {
            const int j = j0 + jj;
            double* Sj = S + (size_t)jj * smem_rows * ES;
            // a. first index of the largest pivot measure in column j, rows j..M-1
            double best = -1.0;
            int bidx = INT_MAX;
            for (int i = jj + tid; i < Mr; i += nthreads) {
                const double* e = Sj + (size_t)i * ES;
                const double v = CPLX ? add_rn(fabs(e[0]), fabs(e[1])) : fabs(e[0]);
                if (v > best || (v == best && i < bidx)) {
                    best = v;
                    bidx = i;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
                if (ov > best || (ov == best && oi < bidx)) {
                    best = ov;
                    bidx = oi;
                }
            }
            if ((tid & 31) == 0) {
                s_val[tid >> 5] = best;
                s_idx[tid >> 5] = bidx;
            }
            __syncthreads();
            double bv = s_val[0];
            int bi = s_idx[0];
            for (int q = 1; q < warps; ++q)
                if (s_val[q] > bv || (s_val[q] == bv && s_idx[q] < bi)) {
                    bv = s_val[q];
                    bi = s_idx[q];
                }
            // A column of NaNs (no comparison succeeds) keeps the diagonal.
            const int pl = bi == INT_MAX ? jj : bi;
            if (tid == 0) d.piv[r0 + j] = r0 + j0 + pl;
            // b. swap rows j and p across the panel's w columns
            if (pl != jj) {
                for (int c = tid; c < w; c += nthreads) {
                    double* x;
                    double* y;
                    if (c >= j0 && c < j0 + sb) {
                        x = S + ((size_t)(c - j0) * smem_rows + jj) * ES;
                        y = S + ((size_t)(c - j0) * smem_rows + pl) * ES;
                    } else {
                        x = P + ((size_t)c * ld + j) * ES;
                        y = P + ((size_t)c * ld + j0 + pl) * ES;
                    }
                    for (int q = 0; q < ES; ++q) {
                        const double tmp = x[q];
                        x[q] = y[q];
                        y[q] = tmp;
                    }
                }
            }
            __syncthreads();
            // c. scale column j below the diagonal, rank-1 update of the
            // sub-panel's columns beyond j
            const Z value = ldz(Sj + (size_t)jj * ES);
            const bool zero = !nonzero(value);
            if (zero && tid == 0) atomicMin(d.singular, r0 + j);
            bool recip;
            Z r;
            if (!CPLX) {
                recip = fabs(value.re) >= kSafeMin;
                r = Z{__ddiv_rn(1.0, value.re), 0.0};
            } else {
                recip = cabs_net(value.re, value.im) >= kSafeMin;
                r = zdiv(Z{1.0, 0.0}, value);
            }
            for (int i = jj + 1 + tid; i < Mr; i += nthreads) {
                Z l = ldz(Sj + (size_t)i * ES);
                if (!zero) {
                    if (!CPLX) l = Z{recip ? mul_rn(l.re, r.re) : __ddiv_rn(l.re, value.re), 0.0};
                    else l = recip ? zmul(l, r) : zdiv(l, value);
                    stz(Sj + (size_t)i * ES, l);
                }
                for (int cc = jj + 1; cc < sb; ++cc) {
                    const Z mult = ldz(S + ((size_t)cc * smem_rows + jj) * ES);
                    if (nonzero(mult)) {
                        double* t = S + ((size_t)cc * smem_rows + i) * ES;
                        stz(t, upd(ldz(t), mult, l));
                    }
                }
            }
            __syncthreads();
        }
        for (int e = tid; e < Mr * sb; e += nthreads) {
            const int i = e % Mr, cc = e / Mr;
            stz(P + ((size_t)(j0 + cc) * ld + j0 + i) * ES, ldz(S + ((size_t)cc * smem_rows + i) * ES));
        }
        const int tc = w - j0 - sb;  // the panel's later columns
        if (tc > 0) {
            // their pivot rows j0 .. j0 + sb - 1: the earlier pivot rows' updates in order
            for (int c = tid; c < tc; c += nthreads) {
                double* col = P + (size_t)(j0 + sb + c) * ld * ES;
                for (int rr = 0; rr < sb; ++rr) {
                    Z t = ldz(col + (size_t)(j0 + rr) * ES);
                    for (int k = 0; k < rr; ++k) {
                        const Z mult = ldz(U + ((size_t)k * kPanelMaxWidth + c) * ES);
                        if (nonzero(mult)) t = upd(t, mult, ldz(S + ((size_t)k * smem_rows + rr) * ES));
                    }
                    stz(col + (size_t)(j0 + rr) * ES, t);
                    stz(U + ((size_t)rr * kPanelMaxWidth + c) * ES, t);
                }
            }
            __syncthreads();
            // every row below: the sb updates in order
            for (int i = sb + tid; i < Mr; i += nthreads) {
                Z l[kPanelSub];
#pragma unroll
                for (int k = 0; k < kPanelSub; ++k) l[k] = k < sb ? ldz(S + ((size_t)k * smem_rows + i) * ES) : Z{0.0, 0.0};
                for (int c = 0; c < tc; ++c) {
                    double* t = P + ((size_t)(j0 + sb + c) * ld + j0 + i) * ES;
                    Z v = ldz(t);
#pragma unroll
                    for (int k = 0; k < kPanelSub; ++k) {
                        if (k < sb) {
                            const Z mult = ldz(U + ((size_t)k * kPanelMaxWidth + c) * ES);
                            if (nonzero(mult)) v = upd(v, mult, l[k]);
                        }
                    }
                    stz(t, v);
                }
            }
        }
        __syncthreads();
    }
}

// The same factorization for one tall panel (thousands of rows), spread over
// every SM: CTA g owns panel rows [g R, (g + 1) R) and keeps them in shared
// memory for the whole panel (the single-CTA kernel re-reads and re-writes
// the trailing panel through L2 for every column, which at 4096 rows is about
// a millisecond per panel). Per column, one grid barrier:
//   before it, every CTA posts its first-largest candidate (value, row) and
//   that row's data, and the owner of row j posts row j (double-buffered by
//   column parity, so one barrier per column suffices);
//   after it, every CTA picks the same pivot p from the candidates (largest
//   measure, lowest row on ties, the diagonal if no comparison succeeds), the
//   owners of rows j and p swap them, and every CTA scales column j and
//   updates its rows with the pivot row.
// Each element sees exactly the single-CTA kernel's operations in the same
// order, so factors and pivots are unchanged (tested bit for bit). The launch
// is cooperative (all CTAs resident); the barrier gives up after 2 s with
// kErrPanelBarrier in the context's error flag, and every CTA then returns.
enum : int { kErrPanelBarrier = 21 };

struct CoopPanelDesc {
    double* a;
    int ld, m, r0, w;
    int* piv;
    int* singular;
    int rows;            // panel rows per CTA
    double* cand_val;    // [2][G]
    int* cand_idx;       // [2][G]
    double* xch;         // [2][G + 1][128]: each CTA's candidate row, then row j
    unsigned* bar;       // arrival count, generation
    int* err;
};

__device__ bool grid_barrier_bounded(unsigned* bar, unsigned nblocks, int* err) {
    __shared__ int s_ok;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g0 = *gen;
        __threadfence();
        bool ok = true;
        if (atomicAdd(bar, 1u) + 1 == nblocks) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const unsigned long long start = global_timer_ns();
            for (uint32_t it = 1; *gen == g0; ++it) {
                if ((it & 255u) == 0) {
                    if (*reinterpret_cast<volatile int*>(err) != 0 || global_timer_ns() - start > kWaitTimeoutNs) {
                        atomicCAS(err, 0, kErrPanelBarrier);
                        ok = false;
                        break;
                    }
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <bool CPLX>
__global__ void __launch_bounds__(256) panel_coop_kernel(const CoopPanelDesc d) {
    constexpr int ES = CPLX ? 2 : 1;
    extern __shared__ double slab[];  // [c][r][q], rows R, columns w
    __shared__ double s_prow[128], s_rowj[128];
    __shared__ double s_val[8];
    __shared__ int s_idx[8], s_own[8];
    __shared__ int s_p, s_owner;
    const int tid = threadIdx.x, G = gridDim.x, g = blockIdx.x;
    const int ld = d.ld, w = d.w, R = d.rows;
    const int M = d.m - d.r0;
    const int rb = g * R, re = min(M, rb + R);
    double* P = d.a + ((size_t)d.r0 * ld + d.r0) * ES;
    auto S = [&](int r, int c) -> double* { return slab + ((size_t)c * R + (r - rb)) * ES; };
    for (int e = tid; e < (re - rb) * w * ES; e += blockDim.x) {
        const int q = e % ES, r = (e / ES) % (re - rb), c = e / (ES * (re - rb));
        S(rb + r, c)[q] = P[((size_t)c * ld + rb + r) * ES + q];
    }
    __syncthreads();
    const int limit = min(M, w);
    for (int j = 0; j < limit; ++j) {
        const int buf = j & 1;
        // a. this CTA's first-largest candidate in column j, rows >= j
        double best = -1.0;
        int bidx = INT_MAX;
        for (int i = max(j, rb) + tid; i < re; i += blockDim.x) {
            const double* e = S(i, j);
            const double v = CPLX ? add_rn(fabs(e[0]), fabs(e[1])) : fabs(e[0]);
            if (v > best || (v == best && i < bidx)) {
                best = v;
                bidx = i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
            if (ov > best || (ov == best && oi < bidx)) {
                best = ov;
                bidx = oi;
            }
        }
        if ((tid & 31) == 0) {
            s_val[tid >> 5] = best;
            s_idx[tid >> 5] = bidx;
        }
        __syncthreads();
        if (tid == 0) {
            double bv = s_val[0];
            int bi = s_idx[0];
            for (int q = 1; q < (int)(blockDim.x >> 5); ++q)
                if (s_val[q] > bv || (s_val[q] == bv && s_idx[q] < bi)) {
                    bv = s_val[q];
                    bi = s_idx[q];
                }
            d.cand_val[buf * G + g] = bv;
            d.cand_idx[buf * G + g] = bi;
            s_p = bi;
        }
        __syncthreads();
        double* slot = d.xch + ((size_t)buf * (G + 1) + g) * 128;
        double* slotj = d.xch + ((size_t)buf * (G + 1) + G) * 128;
        if (s_p != INT_MAX)
            for (int e = tid; e < w * ES; e += blockDim.x) slot[e] = S(s_p, e / ES)[e % ES];
        if (j >= rb && j < re)
            for (int e = tid; e < w * ES; e += blockDim.x) slotj[e] = S(j, e / ES)[e % ES];
        // b. one barrier per column
        if (!grid_barrier_bounded(d.bar, G, d.err)) return;
        // c. the pivot, the same in every CTA: every thread loads candidates
        // (one L2 round trip in parallel), then a block reduction under the
        // same order (larger measure, then lower row).
        {
            double bv = -1.0;
            int bi = INT_MAX, owner = -1;
            for (int q = tid; q < G; q += blockDim.x) {
                const int i = __ldcg(d.cand_idx + buf * G + q);
                const double v = __ldcg(d.cand_val + buf * G + q);
                if (i != INT_MAX && (v > bv || (v == bv && i < bi))) {
                    bv = v;
                    bi = i;
                    owner = q;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                const int oo = __shfl_xor_sync(0xffffffffu, owner, o);
                if (oi != INT_MAX && (ov > bv || (ov == bv && oi < bi))) {
                    bv = ov;
                    bi = oi;
                    owner = oo;
                }
            }
            __syncthreads();  // s_val / s_idx are reused from step a
            if ((tid & 31) == 0) {
                s_val[tid >> 5] = bv;
                s_idx[tid >> 5] = bi;
                s_own[tid >> 5] = owner;
            }
            __syncthreads();
            if (tid == 0) {
                bv = s_val[0];
                bi = s_idx[0];
                owner = s_own[0];
                for (int q = 1; q < (int)(blockDim.x >> 5); ++q)
                    if (s_idx[q] != INT_MAX && (s_val[q] > bv || (s_val[q] == bv && s_idx[q] < bi))) {
                        bv = s_val[q];
                        bi = s_idx[q];
                        owner = s_own[q];
                    }
                if (bi == INT_MAX) {  // no comparison succeeded (NaNs): keep the diagonal
                    bi = j;
                    owner = -1;
                }
                s_p = bi;
                s_owner = owner;
                if (g == 0) d.piv[d.r0 + j] = d.r0 + bi;
            }
            __syncthreads();
        }
        const int p = s_p;
        const double* prow = s_owner >= 0 ? d.xch + ((size_t)buf * (G + 1) + s_owner) * 128 : slotj;
        for (int e = tid; e < w * ES; e += blockDim.x) {
            s_prow[e] = __ldcg(prow + e);
            s_rowj[e] = __ldcg(slotj + e);
        }
        __syncthreads();
        // d. swap rows j and p (each owner writes the other's row)
        if (p != j) {
            if (p >= rb && p < re)
                for (int e = tid; e < w * ES; e += blockDim.x) S(p, e / ES)[e % ES] = s_rowj[e];
            if (j >= rb && j < re)
                for (int e = tid; e < w * ES; e += blockDim.x) S(j, e / ES)[e % ES] = s_prow[e];
        }
        __syncthreads();
        // e. scale column j below the diagonal, then the rank-1 update of columns j+1..w-1
        const int i0 = max(j + 1, rb);
        if (!CPLX) {
            const double value = s_prow[j];
            if (value == 0.0 && g == 0 && tid == 0) atomicMin(d.singular, d.r0 + j);
            const bool recip = fabs(value) >= kSafeMin;
            const double r = __ddiv_rn(1.0, value);
            if (value != 0.0)
                for (int i = i0 + tid; i < re; i += blockDim.x) {
                    double* l = S(i, j);
                    *l = recip ? mul_rn(*l, r) : __ddiv_rn(*l, value);
                }
            __syncthreads();
            const int nr = re - i0, nc = w - j - 1;
            for (int e = tid; e < nr * max(nc, 0); e += blockDim.x) {
                const int i = i0 + e % nr, c = j + 1 + e / nr;
                const double mult = s_prow[c];
                if (mult != 0.0) {
                    double* t = S(i, c);
                    *t = add_rn(*t, mul_rn(-mult, *S(i, j)));
                }
            }
        } else {
            const Z value{s_prow[2 * j], s_prow[2 * j + 1]};
            const bool zero = value.re == 0.0 && value.im == 0.0;
            if (zero && g == 0 && tid == 0) atomicMin(d.singular, d.r0 + j);
            const bool recip = cabs_net(value.re, value.im) >= kSafeMin;
            const Z r = zdiv(Z{1.0, 0.0}, value);
            if (!zero)
                for (int i = i0 + tid; i < re; i += blockDim.x) {
                    double* l = S(i, j);
                    const Z lv{l[0], l[1]};
                    const Z o = recip ? zmul(lv, r) : zdiv(lv, value);
                    l[0] = o.re;
                    l[1] = o.im;
                }
            __syncthreads();
            const int nr = re - i0, nc = w - j - 1;
            for (int e = tid; e < nr * max(nc, 0); e += blockDim.x) {
                const int i = i0 + e % nr, c = j + 1 + e / nr;
                const Z mult{s_prow[2 * c], s_prow[2 * c + 1]};
                if (mult.re == 0.0 && mult.im == 0.0) continue;
                double* t = S(i, c);
                const double* l = S(i, j);
                const Z o = zadd(Z{t[0], t[1]}, zmul(Z{-mult.re, -mult.im}, Z{l[0], l[1]}));
                t[0] = o.re;
                t[1] = o.im;
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < (re - rb) * w * ES; e += blockDim.x) {
        const int q = e % ES, r = (e / ES) % (re - rb), c = e / (ES * (re - rb));
        P[((size_t)c * ld + rb + r) * ES + q] = S(rb + r, c)[q];
    }
}

// Row interchanges rows k <-> piv[k] for k in [k0, k1), applied in increasing
// k (or decreasing, to undo), to columns [c0, c1). One thread per column
// (SwapRows / UnswapRows, Lu.cs:430-478).
struct LaswpDesc {
    double* a;
    int ld, c0, c1;
    const int* piv;
    int k0, k1, reverse;
};

template <bool CPLX>
__global__ void laswp_kernel(const __grid_constant__ Batch<LaswpDesc> b) {
    const LaswpDesc& d = batch_item(b, blockIdx.y);
    constexpr int ES = CPLX ? 2 : 1;
    int c = d.c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.c1) return;
    double* col = d.a + (size_t)c * d.ld * ES;
    for (int s = 0; s < d.k1 - d.k0; ++s) {
        int k = d.reverse ? d.k1 - 1 - s : d.k0 + s;
        int p = d.piv[k];
        if (p != k) {
            for (int q = 0; q < ES; ++q) {
                double tmp = col[(size_t)k * ES + q];
                col[(size_t)k * ES + q] = col[(size_t)p * ES + q];
                col[(size_t)p * ES + q] = tmp;
            }
        }
    }
}

// Triangular block solves, one warp per right-hand side column, w <= 64.
//  kind 0: B := L^-1 B for the unit lower L at t, with the reference's order
//          (x[i] += (-x[p]) * L[i, p] for p = 0..w-2, columns with x[p] == 0
//          skipped; Triangular.SolveLowerUnit, Triangular.cs:26-57, and the
//          complex BlockedLu.cs:312-327).
//  kind 1: X := T^-1 X for the diagonal block of the blocked solves: lower or
//          upper, unit or not, optionally the conjugate transpose of the stored
//          block.
struct TrsmDesc {
    const double* t;
    int ldt;
    double* b;
    int ldb, w, ncols;
    int lower, unit, conj;
};

template <bool CPLX, int KIND>
__global__ void trsm_kernel(const __grid_constant__ Batch<TrsmDesc> bt) {
    const TrsmDesc& d = batch_item(bt, blockIdx.y);
    constexpr int ES = CPLX ? 2 : 1;
    extern __shared__ double sT[];  // effective operator, w x w, ld w: op(i, p)
    const int w = d.w;
    if (d.ncols <= 0 || (int)(blockIdx.x * (blockDim.x >> 5)) >= d.ncols) return;  // nothing for this block
    // Eight loads in flight per thread before their stores.
    for (int e0 = threadIdx.x; e0 < w * w; e0 += 8 * blockDim.x) {
        double re[8], im[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * blockDim.x;
            re[u] = im[u] = 0.0;
            if (e < w * w) {
                const int i = e % w, p = e / w;
                const int si = d.conj ? p : i, sp = d.conj ? i : p;
                const double* src = d.t + ((size_t)sp * d.ldt + si) * ES;
                re[u] = src[0];
                if (CPLX) im[u] = src[1];
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < w * w) {
                sT[(size_t)e * ES] = re[u];
                if (CPLX) sT[(size_t)e * ES + 1] = d.conj ? -im[u] : im[u];
            }
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    for (int c = blockIdx.x * warps + (threadIdx.x >> 5); c < d.ncols; c += gridDim.x * warps) {
        double* x = d.b + (size_t)c * d.ldb * ES;
        Z v[2];
        for (int h = 0; h < 2; ++h) {
            int i = lane + 32 * h;
            v[h].re = i < w ? x[(size_t)i * ES] : 0.0;
            v[h].im = (CPLX && i < w) ? x[(size_t)i * ES + 1] : 0.0;
        }
        const int steps = KIND == 0 ? w - 1 : w;
        for (int s = 0; s < steps; ++s) {
            const bool lower = KIND == 0 ? true : d.lower != 0;
            int p = lower ? s : w - 1 - s;
            int h = p >> 5, src = p & 31;
            if (KIND == 1 && !d.unit) {
                if (lane == src) {
                    if (!CPLX) {
                        v[h].re = __ddiv_rn(v[h].re, sT[(size_t)p * w + p]);
                    } else {
                        Z dg{sT[((size_t)p * w + p) * 2], sT[((size_t)p * w + p) * 2 + 1]};
                        v[h] = zdiv(v[h], dg);
                    }
                }
            }
            double vr = __shfl_sync(0xffffffffu, v[h].re, src);
            double vi = CPLX ? __shfl_sync(0xffffffffu, v[h].im, src) : 0.0;
            if (KIND == 0 && vr == 0.0 && vi == 0.0) continue;
            for (int q = 0; q < 2; ++q) {
                int i = lane + 32 * q;
                bool beyond = lower ? (i > p) : (i < p);
                if (beyond && i < w) {
                    if (!CPLX) {
                        v[q].re = add_rn(v[q].re, mul_rn(-vr, sT[(size_t)p * w + i]));
                    } else {
                        Z tv{sT[((size_t)p * w + i) * 2], sT[((size_t)p * w + i) * 2 + 1]};
                        v[q] = zadd(v[q], zmul(Z{-vr, -vi}, tv));
                    }
                }
            }
        }
        for (int h = 0; h < 2; ++h) {
            int i = lane + 32 * h;
            if (i < w) {
                x[(size_t)i * ES] = v[h].re;
                if (CPLX) x[(size_t)i * ES + 1] = v[h].im;
            }
        }
    }
}

// Triangular substitution in the reference's order. Per right-hand side
// column the reference computes
//   lower, unit:  x[i] += (-x[k]) * L[i,k],                  k = 0..n-2, i > k
//                 (Triangular.SolveLowerUnit; BlockedLu.cs:312-327)
//   upper:        x[k] /= U[k,k]; x[i] += (-x[k]) * U[i,k],  k = n-1..0, i < k
//                 (Triangular.SolveUpper; BlockedLu.cs:329-352)
// and skips every update of a column whose x[k] is zero (its real four-column
// kernels skip only when all four x[k] are zero, which can change nothing but
// the sign of a zero). So each x[i] receives one chain of roundings in the
// order of k, and the chains of different (row, column) pairs are
// independent. The rows are cut into blocks of 32; for each block, in the
// order of k:
//   1. subst_diag_kernel solves the block's own triangle, which completes
//      x[k] for every k of the block;
//   2. subst_update_kernel applies the block's steps to every row beyond it,
//      continuing each row's chain from the value it holds, steps in order.
// Blocking regroups whole chains and never reorders one, so every x[i] sees
// the reference's operations in the reference's order and the solution
// matches bit for bit; step 2, all but about 32/n of the work, runs as a
// register-tiled product on every SM. The adjoint solves accumulate row by
// row in the reference (dot products), an order a right-looking sweep cannot
// reproduce; they stay on the blocked GEMM path.
constexpr int kSubstBlock = 32;

struct SubstDiagDesc {
    const double* f;  // the factors (ld ldf)
    int ldf;
    double* x;  // right-hand sides (ld ldx), overwritten
    int ldx, nrhs;
    int k0, w;  // the block: rows and steps [k0, k0 + w)
};

struct SubstUpdateDesc {
    const double* f;
    int ldf;
    double* x;
    int ldx, nrhs;
    int r0, r1;  // rows updated
    int k0, k1;  // steps applied
    int tiles_m, tile_begin;
};

// x + (-xk) * f with the reference's roundings: a product of two roundings
// per part (no fused multiply-add), then the sum.
template <bool CPLX>
__device__ __forceinline__ Z subst_axpy(Z x, Z nxk, Z f) {
    if (!CPLX) return Z{add_rn(x.re, mul_rn(nxk.re, f.re)), 0.0};
    return zadd(x, zmul(nxk, f));
}

// Step 1: the block's own triangle, one thread per right-hand side column,
// the block's values in registers and its triangle in shared memory (every
// thread reads the same entry at a time: a broadcast).
template <bool CPLX, bool UPPER, bool LDIV = false>
__global__ void __launch_bounds__(128) subst_diag_kernel(const __grid_constant__ Batch<SubstDiagDesc> b) {
    constexpr int B = kSubstBlock;
    constexpr int ES = CPLX ? 2 : 1;
    const SubstDiagDesc& d = batch_item(b, blockIdx.y);
    if ((int)(blockIdx.x * blockDim.x) >= d.nrhs) return;  // whole block idle
    const int w = d.w;
    __shared__ Z t[B][B];  // t[k][i] = F[k0 + i, k0 + k]
    for (int e = threadIdx.x; e < B * B; e += blockDim.x) {
        const int k = e / B, i = e % B;
        Z v{0.0, 0.0};
        if (i < w && k < w) {
            const double* p = d.f + ((size_t)(d.k0 + k) * d.ldf + d.k0 + i) * ES;
            v = Z{p[0], CPLX ? p[1] : 0.0};
        }
        t[k][i] = v;
    }
    __syncthreads();
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.nrhs) return;
    double* x = d.x + ((size_t)col * d.ldx + d.k0) * ES;
    Z v[B];
#pragma unroll
    for (int i = 0; i < B; ++i) {
        v[i] = Z{0.0, 0.0};
        if (i < w) v[i] = Z{x[(size_t)i * ES], CPLX ? x[(size_t)i * ES + 1] : 0.0};
    }
    if (!UPPER) {
#pragma unroll
        for (int k = 0; k < B; ++k) {
            if (k >= w) continue;
            if (LDIV) {
                // An explicit diagonal (Triangular.SolveLower, Triangular.cs:131-150;
                // the adjoint's U^H): x_k /= f_kk first, always for real, and for
                // complex when x_k is not zero (BlockedLu's division rule).
                const Z dg = t[k][k];
                if (!CPLX) v[k].re = __ddiv_rn(v[k].re, dg.re);
                else if (!(v[k].re == 0.0 && v[k].im == 0.0)) v[k] = zdiv(v[k], dg);
            }
            const Z xk = v[k];
            if (k == B - 1 || (xk.re == 0.0 && xk.im == 0.0)) continue;
            const Z nxk{-xk.re, -xk.im};
#pragma unroll
            for (int i = k + 1; i < B; ++i)
                if (i < w) v[i] = subst_axpy<CPLX>(v[i], nxk, t[k][i]);
        }
    } else {
#pragma unroll
        for (int k = B - 1; k >= 0; --k) {
            if (k >= w) continue;
            Z xk = v[k];
            const Z dg = t[k][k];
            if (!CPLX) xk.re = __ddiv_rn(xk.re, dg.re);
            else if (!(xk.re == 0.0 && xk.im == 0.0)) xk = zdiv(xk, dg);
            v[k] = xk;
            if (xk.re == 0.0 && xk.im == 0.0) continue;
            const Z nxk{-xk.re, -xk.im};
#pragma unroll
            for (int i = 0; i < k; ++i) v[i] = subst_axpy<CPLX>(v[i], nxk, t[k][i]);
        }
    }
#pragma unroll
    for (int i = 0; i < B; ++i)
        if (i < w) {
            x[(size_t)i * ES] = v[i].re;
            if (CPLX) x[(size_t)i * ES + 1] = v[i].im;
        }
}

// Asynchronous 16- or 8-byte copies global -> shared; src_bytes 0 fills the
// destination with zeros and reads nothing.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

constexpr int kSubstKC = 16;  // steps per staged round of the update kernel
constexpr int kSubstUpdateSmem = 2 * kSubstKC * (64 + 65) * (int)sizeof(double) * 2;  // two rounds' buffers

// Step 2: rows [r0, r1) of every column take the updates of steps [k0, k1)
// (ascending for the lower factor, descending for the upper), 64 x 64 tiles
// of (row, column) per CTA over a flat grid of every item's tiles. Thread
// (tx, ty) keeps rows tx + 16 r and columns ty + 16 s (r, s < 4) in registers
// from the value x already holds; each round stages 16 steps of the factor
// column and of the solved x[k] in shared memory, the next round's copies in
// flight (cp.async, two buffers) while this one is applied.
template <bool CPLX, bool UPPER>
__global__ void __launch_bounds__(256, 2) subst_update_kernel(const __grid_constant__ Batch<SubstUpdateDesc> b) {
    constexpr int ES = CPLX ? 2 : 1;
    constexpr int KC = kSubstKC;
    int lo = 0, hi = b.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (batch_item(b, mid).tile_begin <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const SubstUpdateDesc& d = batch_item(b, lo);
    const int tile = blockIdx.x - d.tile_begin;
    const int i0 = d.r0 + (tile % d.tiles_m) * 64, c0 = (tile / d.tiles_m) * 64;
    extern __shared__ __align__(16) unsigned char subst_smem[];
    Z* sF = reinterpret_cast<Z*>(subst_smem);  // [2][KC][64]
    Z* sX = sF + 2 * KC * 64;                   // [2][KC][65]
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    if (!CPLX) {
        // 8-byte copies fill only the real parts; the imaginary parts stay 0.
        for (int e = tid; e < 2 * KC * (64 + 65); e += 256) sF[e] = Z{0.0, 0.0};
        __syncthreads();
    }
    auto stage = [&](int q, int buf) {
        const int kq = UPPER ? d.k1 - (q + 1) * KC : d.k0 + q * KC;
        Z* F = sF + buf * KC * 64;
        Z* X = sX + buf * KC * 65;
        for (int e = tid; e < KC * 64; e += 256) {
            const int kk = e >> 6, r = e & 63;
            const int k = kq + kk, i = i0 + r;
            const bool ok = k >= d.k0 && k < d.k1 && i < d.r1;
            const double* p = ok ? d.f + ((size_t)k * d.ldf + i) * ES : d.f;
            if (CPLX) cp_async16(&F[kk * 64 + r], p, ok);
            else cp_async8(&F[kk * 64 + r], p, ok);
        }
        for (int e = tid; e < KC * 64; e += 256) {
            const int kk = e % KC, c = e / KC;
            const int k = kq + kk, col = c0 + c;
            // steps outside [k0, k1) read as zero and are skipped
            const bool ok = k >= d.k0 && k < d.k1 && col < d.nrhs;
            const double* p = ok ? d.x + ((size_t)col * d.ldx + k) * ES : d.x;
            if (CPLX) cp_async16(&X[kk * 65 + c], p, ok);
            else cp_async8(&X[kk * 65 + c], p, ok);
        }
    };
    const int rounds = (d.k1 - d.k0 + KC - 1) / KC;
    stage(0, 0);
    cp_async_commit();
    Z acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int i = i0 + tx + 16 * r, c = c0 + ty + 16 * s;
            acc[r][s] = Z{0.0, 0.0};
            if (i < d.r1 && c < d.nrhs) {
                const double* p = d.x + ((size_t)c * d.ldx + i) * ES;
                acc[r][s] = Z{p[0], CPLX ? p[1] : 0.0};
            }
        }
    for (int q = 0; q < rounds; ++q) {
        if (q + 1 < rounds) {
            stage(q + 1, (q + 1) & 1);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const Z* F = sF + (q & 1) * KC * 64;
        const Z* X = sX + (q & 1) * KC * 65;
#pragma unroll
        for (int j = 0; j < KC; ++j) {
            const int kk = UPPER ? KC - 1 - j : j;
            Z nxk[4];
            bool live[4];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const Z xv = X[kk * 65 + ty + 16 * s];
                live[s] = !(xv.re == 0.0 && xv.im == 0.0);
                nxk[s] = Z{-xv.re, -xv.im};
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const Z fv = F[kk * 64 + tx + 16 * r];
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    if (live[s]) acc[r][s] = subst_axpy<CPLX>(acc[r][s], nxk[s], fv);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int i = i0 + tx + 16 * r, c = c0 + ty + 16 * s;
            if (i < d.r1 && c < d.nrhs) {
                double* p = d.x + ((size_t)c * d.ldx + i) * ES;
                p[0] = acc[r][s].re;
                if (CPLX) p[1] = acc[r][s].im;
            }
        }
}

// min / max |u_jj| over the diagonal (RecordPivotRange, Lu.cs:312-329). The
// values are moduli (never -0), so Math.Min/Math.Max fold to the plain min and
// max unless a NaN is present, which then wins; in that form the fold is
// order-independent and a block reduction gives the reference's result.
template <bool CPLX>
__global__ void pivot_range_kernel(const double* a, int ld, int limit, double* out) {
    __shared__ double s_lo[32], s_hi[32];
    __shared__ int s_nan;
    if (threadIdx.x == 0) s_nan = 0;
    __syncthreads();
    double lo = __longlong_as_double(0x7ff0000000000000ll), hi = 0.0;
    bool nan = false;
    for (int j = threadIdx.x; j < limit; j += blockDim.x) {
        const double* e = a + ((size_t)j * ld + j) * (CPLX ? 2 : 1);
        double v = CPLX ? cabs_net(e[0], e[1]) : fabs(e[0]);
        if (isnan(v)) nan = true;
        lo = fmin(lo, v);
        hi = fmax(hi, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (nan) atomicOr(&s_nan, 1);
    if ((threadIdx.x & 31) == 0) {
        s_lo[threadIdx.x >> 5] = lo;
        s_hi[threadIdx.x >> 5] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            lo = fmin(lo, s_lo[w]);
            hi = fmax(hi, s_hi[w]);
        }
        double qnan = __longlong_as_double(0x7ff8000000000000ll);
        out[0] = s_nan ? qnan : lo;
        out[1] = s_nan ? qnan : hi;
    }
}

__global__ void fill_int_kernel(int* p, int count, int v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) p[i] = v;
}

// ---- launchers ---------------------------------------------------------------

// P B for a solve with few right-hand sides: laswp gives each column one
// thread and n sequential swaps, which leaves the GPU idle when B is narrow.
// Instead one CTA per item replays the swaps on an index array in shared
// memory (row k of P B is row perm[k] of B), and a gather moves every row
// once. The result is the same values in the same places.
struct PermDesc {
    const int* piv;
    int n;
    int* perm;
};
__global__ void build_perm_kernel(const __grid_constant__ Batch<PermDesc> b) {
    const PermDesc& d = batch_item(b, blockIdx.x);
    extern __shared__ int sp[];  // perm [n], pivots [n]
    int* pv = sp + d.n;
    for (int i = threadIdx.x; i < d.n; i += blockDim.x) {
        sp[i] = i;
        pv[i] = d.piv[i];
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < d.n; ++k) {
            const int p = pv[k];
            if (p != k) {
                const int t = sp[k];
                sp[k] = sp[p];
                sp[p] = t;
            }
        }
    __syncthreads();
    for (int i = threadIdx.x; i < d.n; i += blockDim.x) d.perm[i] = sp[i];
}
struct GatherDesc {
    const double* src;
    double* dst;
    int ld, rows, cols;
    const int* perm;
};
template <bool CPLX>
__global__ void gather_rows_kernel(const __grid_constant__ Batch<GatherDesc> b) {
    const GatherDesc& d = batch_item(b, blockIdx.y);
    constexpr int ES = CPLX ? 2 : 1;
    const size_t total = (size_t)d.rows * d.cols;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % d.rows), c = (int)(e / d.rows);
        const double* s = d.src + ((size_t)c * d.ld + d.perm[i]) * ES;
        double* t = d.dst + ((size_t)c * d.ld + i) * ES;
        t[0] = s[0];
        if (CPLX) t[1] = s[1];
    }
}
constexpr int kGatherMaxCols = 128;
constexpr int kGatherMaxRows = 24576;  // perm + pivots in 192 KB of shared memory

// One tall panel over all SMs (panel_coop_kernel), when it has enough rows
// to pay for a barrier per column and every CTA's slab fits shared memory.
constexpr int kCoopPanelRows = 1024;
constexpr size_t kPanelBlockedSmem = 200 * 1024;  // the blocked panel's largest shared-memory footprint

template <bool CPLX>
bool launch_panel_coop(Context& ctx, const PanelFactorDesc& p) {
    constexpr int ES = CPLX ? 2 : 1;
    const int M = p.m - p.r0;
    const int G = ctx.num_sms;
    const int R = (M + G - 1) / G;
    const size_t smem = (size_t)R * p.w * ES * sizeof(double);
    if (smem > 160 * 1024) return false;
    static bool configured[2][64] = {};
    if (!configured[CPLX][ctx.device]) {
        TNS_CUDA(cudaFuncSetAttribute(panel_coop_kernel<CPLX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      160 * 1024));
        configured[CPLX][ctx.device] = true;
    }
    int per_sm = 0;
    TNS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, panel_coop_kernel<CPLX>, 256, smem));
    if (per_sm < 1) return false;
    DBuf scratch(ctx, sizeof(double) * 2 * G + sizeof(int) * 2 * G + sizeof(double) * 2 * (G + 1) * 128 + 64);
    char* base = scratch.as<char>();
    CoopPanelDesc d{};
    d.a = p.a;
    d.ld = p.ld;
    d.m = p.m;
    d.r0 = p.r0;
    d.w = p.w;
    d.piv = p.piv;
    d.singular = p.singular;
    d.rows = R;
    d.xch = reinterpret_cast<double*>(base);
    d.cand_val = d.xch + 2 * (size_t)(G + 1) * 128;
    d.cand_idx = reinterpret_cast<int*>(d.cand_val + 2 * G);
    d.bar = reinterpret_cast<unsigned*>(d.cand_idx + 2 * G);
    d.err = ctx.d_err;
    TNS_CUDA(cudaMemsetAsync(d.bar, 0, 2 * sizeof(unsigned), ctx.stream));
    void* args[] = {&d};
    TNS_CUDA(cudaLaunchCooperativeKernel((const void*)panel_coop_kernel<CPLX>, dim3(G), dim3(256), args, smem,
                                         ctx.stream));
    ctx.kernel_launches++;
    return true;
}

void launch_panels(Context& ctx, bool cplx, std::vector<PanelFactorDesc>& v) {
    if (v.empty()) return;
    // Not in a batch worker: two cooperative panels on concurrent streams
    // could each hold part of the SMs while waiting for the rest.
    if (!ctx.concurrent && v.size() == 1 && v[0].m - v[0].r0 >= kCoopPanelRows && v[0].w <= 64) {
        if (cplx ? launch_panel_coop<true>(ctx, v[0]) : launch_panel_coop<false>(ctx, v[0])) return;
    }
    Batch<PanelFactorDesc> b = make_batch(ctx, v);
    // The blocked panel when every item's sub-panel fits shared memory.
    int rows = 0, width = 0;
    for (auto& p : v) {
        rows = std::max(rows, p.m - p.r0);
        width = std::max(width, p.w);
    }
    const size_t es = cplx ? 2 : 1;
    const size_t smem = sizeof(double) * es * ((size_t)kPanelSub * rows + (size_t)kPanelSub * kPanelMaxWidth);
    if (width <= kPanelMaxWidth && smem <= kPanelBlockedSmem) {
        static bool configured[2][64] = {};
        const int dev = ctx.device >= 0 && ctx.device < 64 ? ctx.device : 0;
        if (!configured[cplx][dev]) {
            if (cplx)
                TNS_CUDA(cudaFuncSetAttribute(panel_blocked_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              kPanelBlockedSmem));
            else
                TNS_CUDA(cudaFuncSetAttribute(panel_blocked_kernel<false>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, kPanelBlockedSmem));
            configured[cplx][dev] = true;
        }
        if (cplx) panel_blocked_kernel<true><<<b.count, 512, smem, ctx.stream>>>(b, rows);
        else panel_blocked_kernel<false><<<b.count, 512, smem, ctx.stream>>>(b, rows);
    } else {
        if (cplx) panel_kernel<true><<<b.count, 512, 0, ctx.stream>>>(b);
        else panel_kernel<false><<<b.count, 512, 0, ctx.stream>>>(b);
    }
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void launch_laswp(Context& ctx, bool cplx, std::vector<LaswpDesc>& v) {
    int maxc = 0;
    std::vector<LaswpDesc> live;
    for (auto& d : v)
        if (d.c1 > d.c0 && d.k1 > d.k0) {
            live.push_back(d);
            maxc = std::max(maxc, d.c1 - d.c0);
        }
    if (live.empty()) return;
    Batch<LaswpDesc> b = make_batch(ctx, live);
    dim3 grid((maxc + 127) / 128, b.count);
    if (cplx) laswp_kernel<true><<<grid, 128, 0, ctx.stream>>>(b);
    else laswp_kernel<false><<<grid, 128, 0, ctx.stream>>>(b);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

template <bool CPLX, int KIND>
void launch_trsm_t(Context& ctx, std::vector<TrsmDesc>& live, int maxcols) {
    // The 64 x 64 complex block needs 64 KB of dynamic shared memory, above
    // the default 48 KB; the attribute is per kernel instance.
    TNS_CUDA(cudaFuncSetAttribute(trsm_kernel<CPLX, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 64 * 16));
    Batch<TrsmDesc> b = make_batch(ctx, live);
    const int threads = 256, warps = threads / 32;
    int per_item = std::max(1, std::min((maxcols + warps - 1) / warps, std::max(1, ctx.num_sms * 4 / (int)live.size())));
    int wmax = 0;
    for (auto& d : live) wmax = std::max(wmax, d.w);
    size_t smem = (size_t)wmax * wmax * (CPLX ? 16 : 8);
    trsm_kernel<CPLX, KIND><<<dim3(per_item, b.count), threads, smem, ctx.stream>>>(b);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void launch_trsm(Context& ctx, bool cplx, int kind, std::vector<TrsmDesc>& v) {
    std::vector<TrsmDesc> live;
    int maxcols = 0;
    for (auto& d : v)
        if (d.ncols > 0 && d.w > (kind == 0 ? 1 : 0)) {
            live.push_back(d);
            maxcols = std::max(maxcols, d.ncols);
        }
    if (live.empty()) return;
    if (cplx) {
        if (kind == 0) launch_trsm_t<true, 0>(ctx, live, maxcols);
        else launch_trsm_t<true, 1>(ctx, live, maxcols);
    } else {
        if (kind == 0) launch_trsm_t<false, 0>(ctx, live, maxcols);
        else launch_trsm_t<false, 1>(ctx, live, maxcols);
    }
}

// One block step of the substitution for every item of a batch: the
// diagonal blocks in one launch, then the updates of all items' tiles in one.
template <bool CPLX, bool UPPER, bool LDIV = false>
void launch_subst_step_t(Context& ctx, std::vector<SubstDiagDesc>& diag, std::vector<SubstUpdateDesc>& upd) {
    if (!diag.empty()) {
        int mr = 0;
        for (auto& d : diag) mr = std::max(mr, d.nrhs);
        Batch<SubstDiagDesc> b = make_batch(ctx, diag);
        subst_diag_kernel<CPLX, UPPER, LDIV><<<dim3((mr + 127) / 128, b.count), 128, 0, ctx.stream>>>(b);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
    }
    if (!upd.empty()) {
        long long total = 0;
        for (auto& u : upd) {
            u.tile_begin = (int)total;
            total += (long long)u.tiles_m * ((u.nrhs + 63) / 64);
        }
        if (total > INT_MAX) fail(TNS_E_ARGUMENT, "triangular solve too large for one launch");
        Batch<SubstUpdateDesc> b = make_batch(ctx, upd);
        static bool configured[64] = {};
        const int dev = ctx.device >= 0 && ctx.device < 64 ? ctx.device : 0;
        if (!configured[dev]) {
            TNS_CUDA(cudaFuncSetAttribute(subst_update_kernel<CPLX, UPPER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kSubstUpdateSmem));
            configured[dev] = true;
        }
        subst_update_kernel<CPLX, UPPER><<<(unsigned)total, 256, kSubstUpdateSmem, ctx.stream>>>(b);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
    }
}

void launch_subst_step(Context& ctx, bool cplx, bool upper, std::vector<SubstDiagDesc>& diag,
                       std::vector<SubstUpdateDesc>& upd, bool lower_divides = false) {
    if (cplx) {
        if (upper) launch_subst_step_t<true, true>(ctx, diag, upd);
        else if (lower_divides) launch_subst_step_t<true, false, true>(ctx, diag, upd);
        else launch_subst_step_t<true, false>(ctx, diag, upd);
    } else {
        if (upper) launch_subst_step_t<false, true>(ctx, diag, upd);
        else if (lower_divides) launch_subst_step_t<false, false, true>(ctx, diag, upd);
        else launch_subst_step_t<false, false>(ctx, diag, upd);
    }
}

// Right-looking substitution of rows [0, n) of every item, in blocks of
// kSubstBlock rows: lower (forward, unit diagonal unless lower_divides) or
// upper (backward, explicit diagonal), the reference's column-oriented order
// (Triangular.SolveLowerUnit / SolveLower / SolveUpper, BlockedLu.SolveLowerUnit /
// SolveUpper). f: the factor (ld ldf), x: the right-hand sides (ld ldx).
struct SubstItem {
    const double* f;
    int ldf;
    double* x;
    int ldx, n, nrhs;
};
// The whole complex substitution in one launch for a few right-hand sides:
// one warp per pair of them (a half-warp each), the pair's columns in shared
// memory, and the factor column each step reads (diagonal included) copied in
// by cp.async kStageAhead steps ahead into a ring of kStageSlots. Step p
// finishes x[p] (the division first where the blocked kernels divide) and,
// unless x[p] is zero, applies subst_axpy(x[i], -x[p], f[i, p]) to every
// later row (lower: rows below, upper: rows above) -- each row's chain in the
// blocked kernels' order, so the same bits, with no launch per 32-row block.
// Real right-hand sides stay on the blocked kernels, which measured as fast
// (n = 512, 8 right-hand sides: 1.1 ms per solve call against 1.25 ms).
// The staged kernels (this one and the left-looking ones below) copy the
// factor column of step s + kStageAhead while step s runs, into a ring of
// kStageSlots columns: far enough ahead that the copies' latency is hidden.
constexpr int kStageSlots = 6;
constexpr int kStageAhead = kStageSlots - 1;
constexpr int kSubstFusedMaxN = 1536;  // complex: 6 slots + 2 columns = 192 KB
constexpr int kSubstFusedMaxRhs = 16;

struct SubstFusedDesc {
    const double* f;
    int ldf;
    double* x;
    int ldx, n, nrhs;
};

template <bool CPLX, bool UPPER, bool LDIV>
__global__ void __launch_bounds__(32) subst_fused_kernel(const __grid_constant__ Batch<SubstFusedDesc> b, int nmax) {
    using E = typename std::conditional<CPLX, double2, double>::type;
    const SubstFusedDesc& d = batch_item(b, blockIdx.y);
    const int n = d.n;
    if ((int)blockIdx.x * 2 >= d.nrhs || n == 0) return;  // the whole warp
    extern __shared__ __align__(16) double ssm[];
    E* slots = reinterpret_cast<E*>(ssm);  // kStageSlots x nmax (nmax: the batch's largest order)
    E* xs = slots + kStageSlots * nmax;    // 2 x nmax
    const int lane = threadIdx.x, L = lane & 15, h = lane >> 4;
    const int col = blockIdx.x * 2 + h;
    const bool active = col < d.nrhs;
    // A half past the last column works on a copy of the pair's first column
    // and never writes it back.
    E* xg = reinterpret_cast<E*>(d.x) + (size_t)(active ? col : blockIdx.x * 2) * d.ldx;
    E* y = xs + h * nmax;
    for (int p = L; p < n; p += 16) y[p] = xg[p];
    // Step s reads column p of the factor over rows [p, n) (lower) or [0, p]
    // (upper), the diagonal at p either way.
    auto issue = [&](int s) {
        if (s < n) {
            const int p = UPPER ? n - 1 - s : s;
            const int r0 = UPPER ? 0 : p, cnt = UPPER ? p + 1 : n - p;
            const E* src = reinterpret_cast<const E*>(d.f) + (size_t)p * d.ldf + r0;
            E* dst = slots + (size_t)(s % kStageSlots) * nmax;
            for (int q = lane; q < cnt; q += 32) {
                if constexpr (CPLX) cp_async16(dst + q, src + q, true);
                else cp_async8(dst + q, src + q, true);
            }
        }
        cp_async_commit();
    };
    for (int q = 0; q < kStageAhead; ++q) issue(q);
    for (int s = 0; s < n; ++s) {
        issue(s + kStageAhead);
        cp_async_wait<kStageAhead>();
        __syncwarp();
        const int p = UPPER ? n - 1 - s : s;
        const int r0 = UPPER ? 0 : p;
        const E* fc = slots + (size_t)(s % kStageSlots) * nmax;  // fc[r - r0] = f[r, p]
        Z xk;
        {
            const E v = y[p];
            if constexpr (CPLX) xk = Z{v.x, v.y};
            else xk = Z{v, 0.0};
        }
        if (UPPER || LDIV) {
            // x_p /= f_pp: always for real; for complex when x_p is not zero.
            const E dv = fc[p - r0];
            if constexpr (!CPLX) {
                xk.re = __ddiv_rn(xk.re, dv);
            } else {
                if (!(xk.re == 0.0 && xk.im == 0.0)) xk = zdiv(xk, Z{dv.x, dv.y});
            }
        }
        if (!(xk.re == 0.0 && xk.im == 0.0)) {
            const Z nxk{-xk.re, -xk.im};
            const int i0 = UPPER ? 0 : p + 1, i1 = UPPER ? p : n;
            auto update = [&](int i, E fv, E xv) {
                if constexpr (CPLX) {
                    const Z r = subst_axpy<true>(Z{xv.x, xv.y}, nxk, Z{fv.x, fv.y});
                    y[i] = make_double2(r.re, r.im);
                } else {
                    y[i] = subst_axpy<false>(Z{xv, 0.0}, nxk, Z{fv, 0.0}).re;
                }
            };
            // Rows are independent within a step: four rows' operands are
            // loaded before their updates.
            int i = i0 + L;
            for (; i + 48 < i1; i += 64) {
                E fv[4], xv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    fv[u] = fc[i + 16 * u - r0];
                    xv[u] = y[i + 16 * u];
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) update(i + 16 * u, fv[u], xv[u]);
            }
            for (; i < i1; i += 16) update(i, fc[i - r0], y[i]);
        }
        // Every lane read x_p above; the divided value goes back only now.
        if ((UPPER || LDIV) && L == 0) {
            if constexpr (CPLX) y[p] = make_double2(xk.re, xk.im);
            else y[p] = xk.re;
        }
        __syncwarp();
    }
    if (active)
        for (int p = L; p < n; p += 16) xg[p] = y[p];
}

template <bool CPLX, bool UPPER, bool LDIV>
void launch_subst_fused(Context& ctx, const std::vector<SubstFusedDesc>& v, int nmax, int pairs) {
    static std::atomic<bool> done[64];
    if (!done[ctx.device].load(std::memory_order_acquire)) {
        TNS_CUDA(cudaFuncSetAttribute(subst_fused_kernel<CPLX, UPPER, LDIV>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
        done[ctx.device].store(true, std::memory_order_release);
    }
    const size_t smem = (size_t)(kStageSlots + 2) * nmax * (CPLX ? 16 : 8);
    subst_fused_kernel<CPLX, UPPER, LDIV><<<dim3(pairs, (unsigned)v.size()), 32, smem, ctx.stream>>>(
        make_batch(ctx, v), nmax);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void substitute(Context& ctx, bool cplx, bool upper, bool lower_divides, const std::vector<SubstItem>& items) {
    {
        // A few complex right-hand sides of orders that fit shared memory: one
        // launch.
        int nmax = 0, rmax = 0;
        bool fits = cplx;
        for (auto& it : items) {
            if (it.n == 0 || it.nrhs == 0) continue;
            nmax = std::max(nmax, it.n);
            rmax = std::max(rmax, it.nrhs);
            fits = fits && it.n <= kSubstFusedMaxN && it.nrhs <= kSubstFusedMaxRhs;
        }
        if (nmax == 0) return;
        if (fits) {
            std::vector<SubstFusedDesc> v;
            for (auto& it : items)
                if (it.n > 0 && it.nrhs > 0) v.push_back(SubstFusedDesc{it.f, it.ldf, it.x, it.ldx, it.n, it.nrhs});
            const int pairs = (rmax + 1) / 2;
            if (upper) launch_subst_fused<true, true, false>(ctx, v, nmax, pairs);
            else if (lower_divides) launch_subst_fused<true, false, true>(ctx, v, nmax, pairs);
            else launch_subst_fused<true, false, false>(ctx, v, nmax, pairs);
            return;
        }
    }
    constexpr int B = kSubstBlock;
    int steps = 0;
    for (auto& it : items)
        if (it.n > 0 && it.nrhs > 0) steps = std::max(steps, (it.n + B - 1) / B);
    for (int s = 0; s < steps; ++s) {
        std::vector<SubstDiagDesc> diag;
        std::vector<SubstUpdateDesc> upd;
        for (auto& it : items) {
            const int n = it.n;
            if (n == 0 || it.nrhs == 0) continue;
            const int blocks = (n + B - 1) / B;
            if (s >= blocks) continue;
            const int k0 = (upper ? blocks - 1 - s : s) * B, w = std::min(B, n - k0);
            diag.push_back(SubstDiagDesc{it.f, it.ldf, it.x, it.ldx, it.nrhs, k0, w});
            const int r0 = upper ? 0 : k0 + w, r1 = upper ? k0 : n;
            if (r1 > r0)
                upd.push_back(SubstUpdateDesc{it.f, it.ldf, it.x, it.ldx, it.nrhs, r0, r1, k0, k0 + w,
                                              (r1 - r0 + 63) / 64, 0});
        }
        launch_subst_step(ctx, cplx, upper, diag, upd, lower_divides);
    }
}

// ---------------------------------------------------------------------------
// Left-looking substitution for the transposed (real) and adjoint (complex)
// solves, whose reference order is an inner product per row: x[i] from the
// x already solved, rows in sequence.
//   FORWARD (U^T): i = 0 .. n-1, the product over rows [0, i) of column i of
//     the factor; backward (L^T / L^H): i = n-1 .. 0, over rows (i, n).
// Real (Triangular.SolveUpperTransposed / SolveLowerTransposed /
// SolveLowerUnitTransposed, Triangular.cs:152-206): x[i] = (x[i] - Dot) / f_ii,
// or x[i] -= Dot on a unit triangle, with ColumnOps.Dot's order: one half-warp
// per right-hand side, lane L holding the 4-lane vector partials
// (netdot_combine), then the scalar tail in order.
// Complex, unit, backward (BlockedLu.SolveLowerUnitAdjoint, BlockedLu.cs:357-373):
// sum = x[i]; sum -= conj(f_ki) x[k] for k ascending; one thread per
// right-hand side.
// ---------------------------------------------------------------------------
template <bool FORWARD, bool UNIT>
__global__ void __launch_bounds__(128) left_subst_real_kernel(const double* __restrict__ f, int ldf, double* x, int ldx,
                                                             int n, int nrhs) {
    const int half = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 4);
    const int L = threadIdx.x & 15, base = threadIdx.x & 16;
    // A half-warp past the last column reads column 0 and drops its results,
    // so that every shuffle sees a converged warp.
    const bool active = half < nrhs;
    double* y = x + (size_t)(active ? half : 0) * ldx;
    constexpr int W = 4;
    for (int step = 0; step < n; ++step) {
        const int i = FORWARD ? step : n - 1 - step;
        const int off = FORWARD ? 0 : i + 1;
        const int len = FORWARD ? i : n - i - 1;
        const double* a = f + (size_t)i * ldf + off;
        const double* yy = y + off;
        const int n16 = (len / (4 * W)) * (4 * W);
        const int n4 = len >= W ? n16 + ((len - n16) / W) * W : 0;
        double total = 0.0;
        if (len >= W) {
            double acc = 0.0;
            for (int p = L; p < n16; p += 16) acc = add_rn(acc, mul_rn(a[p], yy[p]));
            if (L < W)
                for (int p = n16 + L; p < n4; p += W) acc = add_rn(acc, mul_rn(a[p], yy[p]));
            total = netdot_combine(acc, L, base);
        }
        if (L == 0) {
            for (int p = n4; p < len; ++p) total = add_rn(total, mul_rn(a[p], yy[p]));
            if (active) {
                double v = sub_rn(y[i], total);
                if (!UNIT) v = __ddiv_rn(v, f[(size_t)i * ldf + i]);
                y[i] = v;
            }
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(64) left_subst_cplx_unit_back_kernel(const double* __restrict__ f, int ldf, double* x,
                                                                       int ldx, int n, int nrhs) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= nrhs) return;
    double* y = x + (size_t)col * ldx * 2;
    for (int i = n - 1; i >= 0; --i) {
        const double* a = f + (size_t)i * ldf * 2;
        Z sum = zload(y + (size_t)i * 2);
        for (int k = i + 1; k < n; ++k) {
            const Z fk = zload(a + (size_t)k * 2);
            // conj(f) * x in .NET's product order, then sum - product
            const Z p = zmul(Z{fk.re, -fk.im}, zload(y + (size_t)k * 2));
            sum = Z{sub_rn(sum.re, p.re), sub_rn(sum.im, p.im)};
        }
        zstore(y + (size_t)i * 2, sum);
    }
}

// The same two solves with the right-hand sides and the factor in shared
// memory, for the orders that fit: one warp per pair of right-hand sides (a
// half-warp each, both on the same row at each step), the pair's columns kept
// in shared memory, and the factor column a step reads (with its diagonal)
// copied in by cp.async kStageAhead steps ahead into a ring of kStageSlots. A
// step then reads nothing from global memory, and its sums are the kernels' above,
// term for term. Complex: the products conj(f_ki) x[k] of a row are formed by
// the half-warp, then one lane subtracts them in ascending k.
constexpr int kLeftRealMaxN = 3200;  // 6 slots + 2 columns of doubles: 200 KB
constexpr int kLeftCplxMaxN = 1280;  // 6 slots + 2 columns + 2 product rows of complex: 200 KB

template <bool FORWARD, bool UNIT>
__global__ void __launch_bounds__(32) left_subst_real_staged_kernel(const double* __restrict__ f, int ldf, double* x,
                                                                    int ldx, int n, int nrhs) {
    extern __shared__ __align__(16) double lsm[];
    double* slots = lsm;                   // kStageSlots x n
    double* xs = lsm + kStageSlots * n;     // 2 x n
    const int lane = threadIdx.x, L = lane & 15, base = lane & 16, h = lane >> 4;
    const int col = blockIdx.x * 2 + h;
    const bool active = col < nrhs;
    // A half-warp past the last column works on a copy of column 0 and never
    // writes it back, so that every shuffle sees a converged warp.
    double* xg = x + (size_t)(active ? col : 0) * ldx;
    double* y = xs + h * n;
    for (int p = L; p < n; p += 16) y[p] = xg[p];
    // Step s reads column i of the factor over rows [0, i] (forward; the
    // diagonal last) or [i, n) (backward; the diagonal first).
    auto issue = [&](int s) {
        if (s < n) {
            const int i = FORWARD ? s : n - 1 - s;
            const int r0 = FORWARD ? 0 : i, cnt = FORWARD ? i + 1 : n - i;
            const double* src = f + (size_t)i * ldf + r0;
            double* dst = slots + (size_t)(s % kStageSlots) * n;
            for (int p = lane; p < cnt; p += 32) cp_async8(dst + p, src + p, true);
        }
        cp_async_commit();  // empty past the last step, so that every step waits alike
    };
    for (int q = 0; q < kStageAhead; ++q) issue(q);
    constexpr int W = 4;
    for (int s = 0; s < n; ++s) {
        issue(s + kStageAhead);
        cp_async_wait<kStageAhead>();
        __syncwarp();
        const int i = FORWARD ? s : n - 1 - s;
        const int off = FORWARD ? 0 : i + 1;
        const int len = FORWARD ? i : n - i - 1;
        const double* col_f = slots + (size_t)(s % kStageSlots) * n;
        const double* a = FORWARD ? col_f : col_f + 1;
        const double diag = FORWARD ? col_f[i] : col_f[0];
        const double* yy = y + off;
        const int n16 = (len / (4 * W)) * (4 * W);
        const int n4 = len >= W ? n16 + ((len - n16) / W) * W : 0;
        double total = 0.0;
        if (len >= W) {
            double acc = 0.0;
            for (int p = L; p < n16; p += 16) acc = add_rn(acc, mul_rn(a[p], yy[p]));
            if (L < W)
                for (int p = n16 + L; p < n4; p += W) acc = add_rn(acc, mul_rn(a[p], yy[p]));
            total = netdot_combine(acc, L, base);
        }
        if (L == 0) {
            for (int p = n4; p < len; ++p) total = add_rn(total, mul_rn(a[p], yy[p]));
            double v = sub_rn(y[i], total);
            if (!UNIT) v = __ddiv_rn(v, diag);
            y[i] = v;
        }
        __syncwarp();
    }
    if (active)
        for (int p = L; p < n; p += 16) xg[p] = y[p];
}

__global__ void __launch_bounds__(32) left_subst_cplx_unit_back_staged_kernel(const double* __restrict__ f, int ldf,
                                                                              double* x, int ldx, int n, int nrhs) {
    extern __shared__ __align__(16) double lsm[];
    double2* slots = reinterpret_cast<double2*>(lsm);  // kStageSlots x n
    double2* xs = slots + kStageSlots * n;              // 2 x n
    double2* prod = xs + 2 * n;                        // 2 x n
    const int lane = threadIdx.x, L = lane & 15, h = lane >> 4;
    const int col = blockIdx.x * 2 + h;
    const bool active = col < nrhs;
    double2* xg = reinterpret_cast<double2*>(x) + (size_t)(active ? col : 0) * ldx;
    double2* y = xs + h * n;
    double2* pr = prod + h * n;
    for (int p = L; p < n; p += 16) y[p] = xg[p];
    // Step s reads column i = n-1-s of the factor below the diagonal.
    auto issue = [&](int s) {
        if (s < n) {
            const int i = n - 1 - s, cnt = n - i - 1;
            const double2* src = reinterpret_cast<const double2*>(f) + (size_t)i * ldf + i + 1;
            double2* dst = slots + (size_t)(s % kStageSlots) * n;
            for (int p = lane; p < cnt; p += 32) cp_async16(dst + p, src + p, true);
        }
        cp_async_commit();
    };
    for (int q = 0; q < kStageAhead; ++q) issue(q);
    for (int s = 0; s < n; ++s) {
        issue(s + kStageAhead);
        cp_async_wait<kStageAhead>();
        __syncwarp();
        const int i = n - 1 - s, len = n - i - 1;
        const double2* a = slots + (size_t)(s % kStageSlots) * n;
        for (int q = L; q < len; q += 16) {
            const double2 fk = a[q], xk = y[i + 1 + q];
            // conj(f) * x in .NET's product order
            const Z p = zmul(Z{fk.x, -fk.y}, Z{xk.x, xk.y});
            pr[q] = make_double2(p.re, p.im);
        }
        __syncwarp();
        if (L == 0) {
            // Ascending q; eight products loaded ahead of their subtractions.
            double2 sum = y[i];
            int q = 0;
            for (; q + 8 <= len; q += 8) {
                double2 pv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) pv[u] = pr[q + u];
#pragma unroll
                for (int u = 0; u < 8; ++u) sum = make_double2(sub_rn(sum.x, pv[u].x), sub_rn(sum.y, pv[u].y));
            }
            for (; q < len; ++q) {
                const double2 p = pr[q];
                sum = make_double2(sub_rn(sum.x, p.x), sub_rn(sum.y, p.y));
            }
            y[i] = sum;
        }
        __syncwarp();
    }
    if (active)
        for (int p = L; p < n; p += 16) xg[p] = y[p];
}

// Once per kernel and device: the staged kernels take up to 227 KB of
// dynamic shared memory. (One instantiation per kernel: the four share a
// signature, so the flag is keyed on the kernel itself.)
template <auto KERNEL>
void allow_left_smem(int device) {
    static std::atomic<bool> done[64];
    if (done[device].load(std::memory_order_acquire)) return;
    TNS_CUDA(cudaFuncSetAttribute(KERNEL, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    done[device].store(true, std::memory_order_release);
}

// One left-looking solve (see left_subst_real_kernel): real forward U^T
// (unit = false) or backward L^T (unit or not); complex: backward L^H, unit.
void left_substitute(Context& ctx, bool cplx, bool forward, bool unit, const double* f, int ldf, double* x, int ldx,
                     int n, int nrhs) {
    if (n == 0 || nrhs == 0) return;
    const unsigned pairs = (unsigned)((nrhs + 1) / 2);
    if (!cplx && n <= kLeftRealMaxN) {
        const size_t smem = sizeof(double) * (size_t)(kStageSlots + 2) * n;
        if (forward && !unit) {
            allow_left_smem<left_subst_real_staged_kernel<true, false>>(ctx.device);
            left_subst_real_staged_kernel<true, false><<<pairs, 32, smem, ctx.stream>>>(f, ldf, x, ldx, n, nrhs);
        } else if (!forward && unit) {
            allow_left_smem<left_subst_real_staged_kernel<false, true>>(ctx.device);
            left_subst_real_staged_kernel<false, true><<<pairs, 32, smem, ctx.stream>>>(f, ldf, x, ldx, n, nrhs);
        } else if (!forward && !unit) {
            allow_left_smem<left_subst_real_staged_kernel<false, false>>(ctx.device);
            left_subst_real_staged_kernel<false, false><<<pairs, 32, smem, ctx.stream>>>(f, ldf, x, ldx, n, nrhs);
        } else {
            fail(TNS_E_ARGUMENT, "internal: no unit forward transposed solve");
        }
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
        return;
    }
    if (cplx && !forward && unit && n <= kLeftCplxMaxN) {
        const size_t smem = sizeof(double2) * (size_t)(kStageSlots + 4) * n;
        allow_left_smem<left_subst_cplx_unit_back_staged_kernel>(ctx.device);
        left_subst_cplx_unit_back_staged_kernel<<<pairs, 32, smem, ctx.stream>>>(f, ldf, x, ldx, n, nrhs);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
        return;
    }
    if (!cplx) {
        const unsigned grid = (unsigned)((nrhs * 16 + 127) / 128);
        if (forward && !unit) left_subst_real_kernel<true, false><<<grid, 128, 0, ctx.stream>>>(f, ldf, x, ldx, n, nrhs);
        else if (!forward && unit) left_subst_real_kernel<false, true><<<grid, 128, 0, ctx.stream>>>(f, ldf, x, ldx, n, nrhs);
        else if (!forward && !unit) left_subst_real_kernel<false, false><<<grid, 128, 0, ctx.stream>>>(f, ldf, x, ldx, n, nrhs);
        else fail(TNS_E_ARGUMENT, "internal: no unit forward transposed solve");
    } else {
        if (forward || !unit) fail(TNS_E_ARGUMENT, "internal: complex left-looking solves are backward and unit");
        left_subst_cplx_unit_back_kernel<<<(unsigned)((nrhs + 63) / 64), 64, 0, ctx.stream>>>(f, ldf, x, ldx, n, nrhs);
    }
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

inline size_t off(const DMat& a, int i, int j) { return ((size_t)j * a.ld() + i) * (a.cplx ? 2 : 1); }

}  // namespace

// ---------------------------------------------------------------------------

int reference_block_size(int m, int n) { return std::min(m, n) < 1024 ? 32 : 64; }

void getrf_batch(Context& ctx, std::vector<LuItem>& items) {
    if (items.empty()) return;
    const bool cplx = items[0].a->cplx;
    int max_steps = 0;
    for (auto& it : items) {
        int limit = std::min(it.m, it.n);
        if (it.nb < 1) it.nb = reference_block_size(it.m, it.n);
        // The GEMM wants K % 16 == 0 and the panel's pivot-row buffer holds 64.
        it.nb = std::max(16, std::min(64, (it.nb + 15) / 16 * 16));
        fill_int_kernel<<<1, 1, 0, ctx.stream>>>(it.d_sing, 1, INT_MAX);
        ctx.kernel_launches++;
        if (limit == 0) continue;
        // A whole-matrix panel (Lu.cs:244-249) when it fits one panel launch.
        int steps = (it.nb >= limit && it.n <= 64) ? 1 : (limit + it.nb - 1) / it.nb;
        max_steps = std::max(max_steps, steps);
    }
    // LuPhaseTimings (Lu.cs:92-164): CUDA events between the phases of every
    // block step, when the context collects them; a whole-matrix panel is
    // not a blocked loop and records nothing, as in the reference.
    bool blocked = false;
    for (auto& it : items)
        if (std::min(it.m, it.n) > 0 && !(it.nb >= std::min(it.m, it.n) && it.n <= 64)) blocked = true;
    const bool timed = ctx.lu_timing && blocked;
    cudaEvent_t loop_start = nullptr;
    std::vector<cudaEvent_t> marks;
    auto mark = [&]() {
        cudaEvent_t e = ctx.take_event();
        TNS_CUDA(cudaEventRecord(e, ctx.stream));
        marks.push_back(e);
    };
    if (timed) {
        loop_start = ctx.take_event();
        TNS_CUDA(cudaEventRecord(loop_start, ctx.stream));
    }
    for (int k = 0; k < max_steps; ++k) {
        std::vector<PanelFactorDesc> panels;
        std::vector<LaswpDesc> swaps;
        std::vector<TrsmDesc> trsms;
        std::vector<GemmProblem> gemms;
        for (auto& it : items) {
            DMat& a = *it.a;
            const int m = it.m, n = it.n, ld = a.ld();
            const int limit = std::min(m, n);
            if (limit == 0) continue;
            if (it.nb >= limit && n <= 64) {
                if (k == 0) panels.push_back(PanelFactorDesc{a.p, ld, m, 0, n, it.d_piv, it.d_sing});
                continue;
            }
            const int jb = k * it.nb;
            if (jb >= limit) continue;
            const int w = std::min(it.nb, limit - jb);
            panels.push_back(PanelFactorDesc{a.p, ld, m, jb, w, it.d_piv, it.d_sing});
            swaps.push_back(LaswpDesc{a.p, ld, 0, jb, it.d_piv, jb, jb + w, 0});
            if (jb + w >= n) continue;
            swaps.push_back(LaswpDesc{a.p, ld, jb + w, n, it.d_piv, jb, jb + w, 0});
            trsms.push_back(TrsmDesc{a.p + off(a, jb, jb), ld, a.p + off(a, jb, jb + w), ld, w, n - jb - w, 1, 1, 0});
            if (jb + w >= m) continue;
            GemmProblem p{};
            p.A = a.p + off(a, jb + w, jb);
            p.B = a.p + off(a, jb, jb + w);
            p.C = a.p + off(a, jb + w, jb + w);
            p.lda = p.ldb = p.ldc = ld;
            p.M = round_up(m - jb - w, 2);
            p.N = round_up(n - jb - w, 2);
            p.K = w;
            p.alpha_re = -1.0;
            p.beta_re = 1.0;
            p.work = (long long)(m - jb - w) * (n - jb - w) * w;
            gemms.push_back(p);
        }
        if (timed) mark();
        launch_panels(ctx, cplx, panels);
        if (timed) mark();
        launch_laswp(ctx, cplx, swaps);
        if (timed) mark();
        launch_trsm(ctx, cplx, 0, trsms);
        if (timed) mark();
        if (!gemms.empty()) gemm_grouped(ctx, gemms, cplx);
        if (timed) mark();
    }
    if (timed) {
        cudaEvent_t loop_end = ctx.take_event();
        TNS_CUDA(cudaEventRecord(loop_end, ctx.stream));
        TNS_CUDA(cudaStreamSynchronize(ctx.stream));
        auto ms = [](cudaEvent_t a, cudaEvent_t b) {
            float v = 0.f;
            TNS_CUDA(cudaEventElapsedTime(&v, a, b));
            return (double)v;
        };
        for (size_t q = 0; q + 5 <= marks.size(); q += 5) {
            ctx.lu_panel_ms += ms(marks[q], marks[q + 1]);
            ctx.lu_swaps_ms += ms(marks[q + 1], marks[q + 2]);
            ctx.lu_triangular_ms += ms(marks[q + 2], marks[q + 3]);
            ctx.lu_gemm_ms += ms(marks[q + 3], marks[q + 4]);
        }
        ctx.lu_total_ms += ms(loop_start, loop_end);
        ctx.lu_block_steps += max_steps;
        ctx.lu_factorizations += (long long)items.size();
        for (cudaEvent_t e : marks) ctx.event_pool.push_back(e);
        ctx.event_pool.push_back(loop_start);
        ctx.event_pool.push_back(loop_end);
    }
}

void getrs_batch(Context& ctx, std::vector<SolveItem>& items, bool adjoint) {
    if (items.empty()) return;
    const bool cplx = items[0].lu->cplx;
    std::vector<DMat> herm;  // conjugate transposes for the complex adjoint solves
    if (adjoint && cplx) {
        herm.reserve(items.size());
        for (auto& it : items) {
            herm.emplace_back(ctx, it.lu->cols, it.lu->rows, cplx, "the conjugate transpose of the factors");
            conj_transpose(ctx, herm.back(), *it.lu);
        }
    }
    if (!adjoint) {
        // P B, then L (unit lower) forward and U backward by substitution in
        // the reference's order (Lu.Solve, Lu.cs:336-351; BlockedLu.Solve,
        // BlockedLu.cs:105-118): the result matches the reference bit for bit.
        std::vector<LaswpDesc> swaps;
        std::vector<SolveItem*> narrow;
        for (auto& it : items) {
            int n = it.lu->rows;
            if (n == 0 || it.nrhs == 0) continue;
            if (it.nrhs < kGatherMaxCols && n <= kGatherMaxRows) narrow.push_back(&it);
            else swaps.push_back(LaswpDesc{it.b->p, it.b->ld(), 0, it.nrhs, it.d_piv, 0, n, 0});
        }
        launch_laswp(ctx, cplx, swaps);
        if (!narrow.empty()) {
            size_t total = 0;
            int maxn = 0;
            for (auto* it : narrow) {
                total += (size_t)it->lu->rows;
                maxn = std::max(maxn, it->lu->rows);
            }
            DBuf perms(ctx, sizeof(int) * total);
            std::vector<DMat> tmp;
            tmp.reserve(narrow.size());
            std::vector<PermDesc> pd;
            std::vector<GatherDesc> gd;
            size_t off = 0;
            long long maxe = 0;
            for (auto* it : narrow) {
                const int n = it->lu->rows;
                tmp.emplace_back(ctx, it->b->rows, it->b->cols, cplx, "the permuted right-hand sides");
                pd.push_back(PermDesc{it->d_piv, n, perms.as<int>() + off});
                gd.push_back(GatherDesc{it->b->p, tmp.back().p, it->b->ld(), n, it->nrhs, perms.as<int>() + off});
                off += (size_t)n;
                maxe = std::max(maxe, (long long)n * it->nrhs);
            }
            Batch<PermDesc> bp = make_batch(ctx, pd);
            const size_t smem = sizeof(int) * 2 * (size_t)maxn;
            static bool configured[64] = {};
            if (!configured[ctx.device]) {
                TNS_CUDA(cudaFuncSetAttribute(build_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)(sizeof(int) * 2 * kGatherMaxRows)));
                configured[ctx.device] = true;
            }
            build_perm_kernel<<<bp.count, 256, smem, ctx.stream>>>(bp);
            TNS_CUDA(cudaGetLastError());
            Batch<GatherDesc> bg = make_batch(ctx, gd);
            const dim3 grid((unsigned)std::min<long long>((maxe + 255) / 256, ctx.num_sms * 8), bg.count);
            if (cplx) gather_rows_kernel<true><<<grid, 256, 0, ctx.stream>>>(bg);
            else gather_rows_kernel<false><<<grid, 256, 0, ctx.stream>>>(bg);
            TNS_CUDA(cudaGetLastError());
            ctx.kernel_launches += 2;
            // back into B, only the solve's nrhs columns (contiguous: ld = rows_p)
            for (size_t q = 0; q < narrow.size(); ++q)
                TNS_CUDA(cudaMemcpyAsync(narrow[q]->b->p, tmp[q].p,
                                         (size_t)narrow[q]->b->ld() * narrow[q]->nrhs * narrow[q]->b->esz(),
                                         cudaMemcpyDeviceToDevice, ctx.stream));
        }
        std::vector<SubstItem> subst;
        for (auto& it : items)
            if (it.lu->rows > 0 && it.nrhs > 0)
                subst.push_back(SubstItem{it.lu->p, it.lu->ld(), it.b->p, it.b->ld(), it.lu->rows, it.nrhs});
        substitute(ctx, cplx, false, false, subst);  // L, unit diagonal, forward
        substitute(ctx, cplx, true, false, subst);   // U, backward
        return;
    }
    // The adjoint in the reference's order (Lu.SolveTransposed, Lu.cs:364-378;
    // BlockedLu.SolveAdjoint, BlockedLu.cs:130-141): U^H forward, then L^H
    // backward, then the interchanges undone.
    for (size_t q = 0; q < items.size(); ++q) {
        auto& it = items[q];
        const int n = it.lu->rows;
        if (n == 0 || it.nrhs == 0) continue;
        if (!cplx) {
            // Both by inner products in ColumnOps.Dot's order.
            left_substitute(ctx, false, true, false, it.lu->p, it.lu->ld(), it.b->p, it.b->ld(), n, it.nrhs);
            left_substitute(ctx, false, false, true, it.lu->p, it.lu->ld(), it.b->p, it.b->ld(), n, it.nrhs);
        } else {
            // U^H: its sums run in ascending k, which a right-looking sweep over
            // the conjugate transpose reproduces; L^H: ascending k inside a
            // backward sweep, one inner product per row.
            std::vector<SubstItem> fwd{SubstItem{herm[q].p, herm[q].ld(), it.b->p, it.b->ld(), n, it.nrhs}};
            substitute(ctx, true, false, true, fwd);
            left_substitute(ctx, true, false, true, it.lu->p, it.lu->ld(), it.b->p, it.b->ld(), n, it.nrhs);
        }
    }
    if (adjoint) {
        std::vector<LaswpDesc> swaps;
        for (auto& it : items) {
            int n = it.lu->rows;
            if (n == 0 || it.nrhs == 0) continue;
            swaps.push_back(LaswpDesc{it.b->p, it.b->ld(), 0, it.nrhs, it.d_piv, 0, n, 1});
        }
        launch_laswp(ctx, cplx, swaps);
    }
}

LuResult getrf(Context& ctx, DMat& a, int m, int n, int nb, int* d_piv) {
    LuResult res;
    int limit = std::min(m, n);
    if (limit == 0) return res;
    DBuf flags(ctx, sizeof(int) + 2 * sizeof(double) + 8);
    int* d_sing = flags.as<int>();
    double* d_range = reinterpret_cast<double*>(flags.as<char>() + 8);
    std::vector<LuItem> items{LuItem{&a, m, n, nb, d_piv, d_sing}};
    getrf_batch(ctx, items);
    if (a.cplx)
        pivot_range_kernel<true><<<1, 256, 0, ctx.stream>>>(a.p, a.ld(), limit, d_range);
    else
        pivot_range_kernel<false><<<1, 256, 0, ctx.stream>>>(a.p, a.ld(), limit, d_range);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
    int h_sing = INT_MAX;
    double h_range[2];
    TNS_CUDA(cudaMemcpyAsync(&h_sing, d_sing, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    TNS_CUDA(cudaMemcpyAsync(h_range, d_range, sizeof(h_range), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    res.singular_column = h_sing == INT_MAX ? -1 : h_sing;
    res.smallest_pivot = h_range[0];
    res.largest_pivot = h_range[1];
    return res;
}

void getrs(Context& ctx, const DMat& lu, const int* d_piv, DMat& b, int nrhs, bool adjoint) {
    std::vector<SolveItem> items{SolveItem{&lu, d_piv, &b, nrhs}};
    getrs_batch(ctx, items, adjoint);
}

void getrs_free_order(Context& ctx, const DMat& lu, const int* d_piv, DMat& b, int nrhs, bool adjoint) {
    const int n = lu.rows;
    if (n == 0 || nrhs == 0) return;
    const bool cplx = lu.cplx;
    const size_t es = cplx ? 2 : 1;
    constexpr int bs = 64;
    const int blocks = (n + bs - 1) / bs;
    const int ld = lu.ld(), ldb = b.ld();
    DMat herm;  // the conjugate transpose, for the adjoint's GEMM updates
    if (adjoint) {
        herm = DMat(ctx, lu.cols, lu.rows, cplx, "the conjugate transpose of the factors");
        conj_transpose(ctx, herm, lu);
    }
    const double* G = adjoint ? herm.p : lu.p;
    const int ldg = adjoint ? herm.ld() : ld;
    auto update = [&](const double* A, const double* X, double* C, int rows, int k) {
        if (rows <= 0) return;
        GemmProblem p{};
        p.A = A;
        p.B = X;
        p.C = C;
        p.lda = ldg;
        p.ldb = p.ldc = ldb;
        p.M = round_up(rows, 2);
        p.N = round_up(nrhs, 2);
        p.K = round_up(k, 16);
        p.alpha_re = -1.0;
        p.beta_re = 1.0;
        std::vector<GemmProblem> g{p};
        gemm_grouped(ctx, g, cplx);
    };
    if (!adjoint && d_piv) {
        std::vector<LaswpDesc> sw{LaswpDesc{b.p, ldb, 0, nrhs, d_piv, 0, n, 0}};
        launch_laswp(ctx, cplx, sw);
    }
    // Forward: L (unit) or U^H (explicit diagonal), then the rows below.
    for (int kb = 0; kb < blocks; ++kb) {
        const int k0 = kb * bs, w = std::min(bs, n - k0);
        std::vector<TrsmDesc> d{TrsmDesc{lu.p + ((size_t)k0 * ld + k0) * es, ld, b.p + (size_t)k0 * es, ldb, w, nrhs, 1,
                                         adjoint ? 0 : 1, adjoint ? 1 : 0}};
        launch_trsm(ctx, cplx, 1, d);
        update(G + ((size_t)k0 * ldg + k0 + w) * es, b.p + (size_t)k0 * es, b.p + (size_t)(k0 + w) * es, n - k0 - w, w);
    }
    // Backward: U (explicit diagonal) or L^H (unit), then the rows above.
    for (int kb = blocks - 1; kb >= 0; --kb) {
        const int k0 = kb * bs, w = std::min(bs, n - k0);
        std::vector<TrsmDesc> d{TrsmDesc{lu.p + ((size_t)k0 * ld + k0) * es, ld, b.p + (size_t)k0 * es, ldb, w, nrhs, 0,
                                         adjoint ? 1 : 0, adjoint ? 1 : 0}};
        launch_trsm(ctx, cplx, 1, d);
        update(G + ((size_t)k0 * ldg) * es, b.p + (size_t)k0 * es, b.p, k0, w);
    }
    if (adjoint && d_piv) {
        std::vector<LaswpDesc> sw{LaswpDesc{b.p, ldb, 0, nrhs, d_piv, 0, n, 1}};
        launch_laswp(ctx, cplx, sw);
    }
}

void solve_triangular(Context& ctx, TriangularKind kind, const DMat& f, DMat& b, int nrhs) {
    const int n = f.rows;
    if (n == 0 || nrhs == 0) return;
    const bool cplx = f.cplx;
    std::vector<SubstItem> it{SubstItem{f.p, f.ld(), b.p, b.ld(), n, nrhs}};
    switch (kind) {
        case TriangularKind::kUpper: substitute(ctx, cplx, true, false, it); break;
        case TriangularKind::kLowerUnit: substitute(ctx, cplx, false, false, it); break;
        case TriangularKind::kLower:
            if (cplx) fail(TNS_E_ARGUMENT, "internal: no complex explicit-diagonal lower solve");
            substitute(ctx, false, false, true, it);
            break;
        case TriangularKind::kUpperTransposed:
            if (!cplx) {
                left_substitute(ctx, false, true, false, f.p, f.ld(), b.p, b.ld(), n, nrhs);
            } else {
                DMat h(ctx, f.cols, f.rows, true, "the conjugate transpose of a triangle");
                conj_transpose(ctx, h, f);
                std::vector<SubstItem> fw{SubstItem{h.p, h.ld(), b.p, b.ld(), n, nrhs}};
                substitute(ctx, true, false, true, fw);
            }
            break;
        case TriangularKind::kLowerTransposed:
            if (cplx) fail(TNS_E_ARGUMENT, "internal: no complex explicit-diagonal lower solve");
            left_substitute(ctx, false, false, false, f.p, f.ld(), b.p, b.ld(), n, nrhs);
            break;
        case TriangularKind::kLowerUnitTransposed:
            left_substitute(ctx, cplx, false, true, f.p, f.ld(), b.p, b.ld(), n, nrhs);
            break;
    }
}

// ---------------------------------------------------------------------------
// The precision form of the solve (no counterpart in the reference, whose
// solves are FP64 throughout: Lu.Factor + Lu.Solve, Lu.cs:230-351).
//
// Factorization. Right-looking in blocks of 512 columns: the 512-wide panel
// is factored by getrf_batch (its own 64-column steps, FP64 panels and DMMA
// updates), its row interchanges are applied either side, U12 := L11^-1 A12
// by 64-row triangular blocks and DMMA updates, and the trailing update
// A22 -= L21 U12 -- almost all of the (2/3) n^3 flops -- runs on the
// split-precision product (8-bit residues on the tensor cores) with depth
// 512. Its precision is set by the moduli: the integer images keep t bits
// (26 with 8 moduli, 49 with 14), so the factors are those of A + dA with
// |dA| about 2^-t of the operands' scales per update.
// Refinement. x = U^-1 L^-1 P b, then r = b - A x in FP64 (DMMA GEMM),
// d = U^-1 L^-1 P r, x += d, until the normwise backward error
// max_j |r_j|_inf / (|A|_inf |x_j|_inf + |b_j|_inf) reaches 4 u (u = 2^-53),
// stops halving, or max_iter steps are done. The refinement converges while
// kappa(A) 2^-t is well below 1 (each step multiplies the error by about
// that); with moduli = 0 the moduli are chosen from the condition estimate
// kappa_1 of the first (8-moduli) factors so that t >= log2(kappa_1) + 7,
// refactoring once if that needs more than 8.

namespace {

// A non-owning view of the rows x cols block of `a` at (i, j): same leading
// dimension, and it frees nothing.
DMat block_view(const DMat& a, int i, int j, int rows, int cols) {
    DMat v;
    v.p = const_cast<double*>(a.at(i, j));
    v.rows = rows;
    v.cols = cols;
    v.rows_p = a.rows_p;
    v.cols_p = cols;
    v.cplx = a.cplx;
    return v;
}

__global__ void add_offset_kernel(int* p, int count, int v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) p[i] += v;
}

// dst := f * src for a rows x cols block (es doubles per element).
__global__ void scaled_block_copy_kernel(double* dst, int ldd, const double* src, int lds, int rows, int cols,
                                         double f, int es) {
    const size_t h = (size_t)rows * es;
    const size_t total = h * cols;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t r = e % h, c = e / h;
        dst[c * ldd * es + r] = mul_rn(src[c * lds * es + r], f);
    }
}

// out[j] = max_i |x_ij| (complex: the modulus), one warp per column.
template <bool CPLX>
__global__ void col_absmax_kernel(const double* x, int ld, int rows, int cols, double* out) {
    const int j = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (j >= cols) return;
    double m = 0.0;
    for (int i = lane; i < rows; i += 32) {
        const double v = CPLX ? hypot(x[((size_t)j * ld + i) * 2], x[((size_t)j * ld + i) * 2 + 1])
                              : fabs(x[(size_t)j * ld + i]);
        m = fmax(m, v);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) out[j] = m;
}

std::vector<double> col_absmax(Context& ctx, const DMat& x) {
    DBuf buf(ctx, sizeof(double) * std::max(1, x.cols));
    const int warps = 8;
    if (x.cplx)
        col_absmax_kernel<true><<<(x.cols + warps - 1) / warps, 32 * warps, 0, ctx.stream>>>(x.p, x.ld(), x.rows,
                                                                                          x.cols, buf.as<double>());
    else
        col_absmax_kernel<false><<<(x.cols + warps - 1) / warps, 32 * warps, 0, ctx.stream>>>(x.p, x.ld(), x.rows,
                                                                                           x.cols, buf.as<double>());
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
    std::vector<double> out(x.cols);
    TNS_CUDA(cudaMemcpyAsync(out.data(), buf.p, sizeof(double) * x.cols, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    return out;
}

constexpr int kMixedOuter = 512;  // depth of the split-precision trailing updates

// Below a factored panel of w columns at column j: U12 := L11^-1 A12 (64-row
// unit-lower blocks, DMMA updates below each), then A22 -= L21 U12 on the
// split-precision product with `moduli` moduli.
void mixed_trailing(Context& ctx, DMat& a, int j, int w, int moduli) {
    const int n = a.rows, ld = a.ld();
    const bool cplx = a.cplx;
    const int es = cplx ? 2 : 1;
    const int rest = n - j - w;
    // U12 := L11^-1 A12: 64-row unit-lower blocks, DMMA updates below each.
    for (int b0 = 0; b0 < w; b0 += 64) {
        const int bw = std::min(64, w - b0);
        std::vector<TrsmDesc> t{TrsmDesc{a.at(j + b0, j + b0), ld, a.at(j + b0, j + w), ld, bw, rest, 1, 1, 0}};
        launch_trsm(ctx, cplx, 1, t);
        if (b0 + bw < w) {
            GemmProblem p{};
            p.A = a.at(j + b0 + bw, j + b0);
            p.B = a.at(j + b0, j + w);
            p.C = a.at(j + b0 + bw, j + w);
            p.lda = p.ldb = p.ldc = ld;
            p.M = round_up(w - b0 - bw, 2);
            p.N = round_up(rest, 2);
            p.K = round_up(bw, 16);
            p.alpha_re = -1.0;
            p.beta_re = 1.0;
            p.work = (long long)(w - b0 - bw) * rest * bw;
            std::vector<GemmProblem> g{p};
            gemm_grouped(ctx, g, cplx);
        }
    }
    // A22 -= L21 U12 on the split-precision product: C += (-L21) U12.
    DMat negl(ctx, rest, w, cplx, "the negated L21 block of a mixed-precision factorization");
    {
        const size_t total = (size_t)rest * es * w;
        const int grid = (int)std::min<size_t>((total + 255) / 256, (size_t)ctx.num_sms * 16);
        scaled_block_copy_kernel<<<grid, 256, 0, ctx.stream>>>(negl.p, negl.ld(), a.at(j + w, j), ld, rest, w,
                                                              -1.0, es);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
    }
    DMat u12 = block_view(a, j, j + w, w, rest);
    DMat a22 = block_view(a, j + w, j + w, rest, rest);
    std::vector<SplitProduct> sp{SplitProduct{&negl, &u12, &a22, 1.0}};
    gemm_split_batch(ctx, sp, moduli);
}

}  // namespace

void getrf_mixed(Context& ctx, DMat& a, int* d_piv, int moduli) {
    const int n = a.rows, ld = a.ld();
    const bool cplx = a.cplx;
    const int es = cplx ? 2 : 1;
    const int blocks = (n + kMixedOuter - 1) / kMixedOuter;
    DBuf sing(ctx, sizeof(int) * std::max(1, blocks));
    for (int q = 0; q < blocks; ++q) {
        const int j = q * kMixedOuter, w = std::min(kMixedOuter, n - j);
        DMat panel = block_view(a, j, j, n - j, w);
        int* piv = d_piv + j;  // rows relative to row j until the offset below
        {
            std::vector<LuItem> items{LuItem{&panel, n - j, w, 64, piv, sing.as<int>() + q}};
            getrf_batch(ctx, items);
        }
        std::vector<LaswpDesc> sw;
        double* rowj = a.p + (size_t)j * es;
        if (j > 0) sw.push_back(LaswpDesc{rowj, ld, 0, j, piv, 0, w, 0});
        if (j + w < n) sw.push_back(LaswpDesc{rowj, ld, j + w, n, piv, 0, w, 0});
        launch_laswp(ctx, cplx, sw);
        add_offset_kernel<<<(w + 255) / 256, 256, 0, ctx.stream>>>(piv, w, j);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
        if (j + w >= n) break;
        mixed_trailing(ctx, a, j, w, moduli);
    }
    std::vector<int> flags(blocks);
    TNS_CUDA(cudaMemcpyAsync(flags.data(), sing.p, sizeof(int) * blocks, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    for (int q = 0; q < blocks; ++q)
        if (flags[q] != INT_MAX)
            fail(TNS_E_SINGULAR, "The low-precision factorization met an exactly zero pivot at column " +
                                     std::to_string(q * kMixedOuter + flags[q]) + ".");
}

namespace {

// The precision form with partial pivoting (the fallback of gesv_mixed).
void gesv_mixed_pivoted(Context& ctx, const DMat& a, const DMat& b, DMat& x, int moduli, int max_iter,
                        MixedInfo& info) {
    const int n = a.rows, nrhs = b.cols;
    const bool cplx = a.cplx;
    info = MixedInfo{};
    info.pivoting = 1;
    DMat f(ctx, n, n, cplx, "the low-precision factors");
    DBuf piv(ctx, sizeof(int) * (size_t)std::max(1, n));
    auto factor = [&](int m) {
        copy_dmat(ctx, f, a);
        getrf_mixed(ctx, f, piv.as<int>(), m);
        info.factorizations++;
        info.moduli = m;
    };
    factor(moduli > 0 ? moduli : 8);
    const double anorm1 = norm1(ctx, a);
    const NormestResult est = normest_lu_inverse(ctx, f, piv.as<int>(), 2, 5, 20260915, true);
    info.rcond = (anorm1 > 0.0 && est.value > 0.0) ? 1.0 / (anorm1 * est.value) : 0.0;
    if (moduli == 0) {
        const double kappa = info.rcond > 0.0 ? 1.0 / info.rcond : 1e300;
        const int need = (int)std::ceil(std::log2(std::max(1.0, kappa))) + 7;
        const int depth = cplx ? 2 * kMixedOuter : kMixedOuter;
        int m = info.moduli;
        while (m < 22 && split_integer_bits(m, depth) < need) ++m;
        if (m > info.moduli) {
            factor(m);
            const NormestResult again = normest_lu_inverse(ctx, f, piv.as<int>(), 2, 5, 20260915, true);
            info.rcond = (anorm1 > 0.0 && again.value > 0.0) ? 1.0 / (anorm1 * again.value) : 0.0;
        }
    }
    x = DMat(ctx, n, nrhs, cplx, "the solution");
    copy_dmat(ctx, x, b);
    // The precision form's solves have no reference order to keep: blocked
    // triangular solves with DMMA updates.
    getrs_free_order(ctx, f, piv.as<int>(), x, nrhs, false);
    const double ainf = norminf(ctx, a);
    const std::vector<double> bmax = col_absmax(ctx, b);
    DMat r(ctx, n, nrhs, cplx, "the refinement residual");
    double prev = INFINITY;
    for (int it = 0;; ++it) {
        copy_dmat(ctx, r, b);
        std::vector<GemmProblem> g{make_gemm(a, x, r, -1.0, 0.0, 1.0, 0.0)};
        gemm_grouped(ctx, g, cplx);
        const std::vector<double> rmax = col_absmax(ctx, r), xmax = col_absmax(ctx, x);
        double berr = 0.0;
        for (int j = 0; j < nrhs; ++j) {
            const double den = ainf * xmax[j] + bmax[j];
            berr = std::max(berr, den > 0.0 ? rmax[j] / den : (rmax[j] > 0.0 ? INFINITY : 0.0));
        }
        info.backward_error = berr;
        if (berr <= 4.0 * 1.1102230246251565e-16 || it >= max_iter || !(berr < 0.5 * prev)) break;
        prev = berr;
        getrs_free_order(ctx, f, piv.as<int>(), r, nrhs, false);
        std::vector<EwDesc> add{ew_add_scaled(x, r, 1.0)};
        ew_batch(ctx, add);
        info.iterations++;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// The precision form without row interchanges. Random butterfly transforms
// (Parker, 1995; Baboulin, Dongarra, Herrmann and Tomov, 2013) make Gaussian
// elimination without pivoting stable with high probability: A x = b becomes
// (T A S) y = T b, x = S y, with T = T2 T1 and S = S1 S2 recursive
// butterflies of depth 2. A butterfly of order 2h is
// B = (1/sqrt 2) [[R0, R1], [R0, -R1]], R0 and R1 diagonal with entries
// exp(r / 10), r uniform in [-1/2, 1/2]; level 1 is one butterfly of the
// whole order N, level 2 two of order N/2. T_i = B_i^T act on rows, S_i = B_i
// on columns. The order is padded to N = round_up(n, 4) with an identity
// block. Without pivot searches the panels are a 64 x 64 diagonal block, a
// right triangular solve and DMMA updates, so nothing serialises on one SM
// per column; the refinement's residuals use A itself in FP64.
// ---------------------------------------------------------------------------
namespace {

constexpr double kInvSqrt2 = 0.70710678118654752440;
constexpr int kNopivBlock = 64;
constexpr int kNopivLd = kNopivBlock + 1;  // shared-memory column stride of the 64 x 64 blocks

template <bool CPLX>
__device__ __forceinline__ Z load_el(const double* p) {
    return CPLX ? Z{p[0], p[1]} : Z{p[0], 0.0};
}
template <bool CPLX>
__device__ __forceinline__ void store_el(double* p, Z v) {
    p[0] = v.re;
    if (CPLX) p[1] = v.im;
}
// acc - x y
template <bool CPLX>
__device__ __forceinline__ Z sub_prod(Z acc, Z x, Z y) {
    if (!CPLX) return Z{sub_rn(acc.re, mul_rn(x.re, y.re)), 0.0};
    const Z p = zmul(x, y);
    return Z{sub_rn(acc.re, p.re), sub_rn(acc.im, p.im)};
}
template <bool CPLX>
__device__ __forceinline__ Z div_el(Z x, Z y) {
    return CPLX ? zdiv(x, y) : Z{__ddiv_rn(x.re, y.re), 0.0};
}

// One butterfly level on the rows of an N x cols panel (ld elements): the
// pairs (i, i + h) of every segment of 2h rows. kind 0: B^T,
// (u, v) -> (d_i (u + v), d_{i+h} (u - v)) / sqrt 2; kind 1: B,
// (u, v) -> (d_i u + d_{i+h} v, d_i u - d_{i+h} v) / sqrt 2.
template <bool CPLX>
__global__ void butterfly_rows_kernel(double* a, int ld, int n, int cols, int h, const double* d, int kind) {
    constexpr int ES = CPLX ? 2 : 1;
    const int half = n / 2;
    const size_t total = (size_t)half * cols;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(e % half), c = (int)(e / half);
        const int i = (q / h) * 2 * h + q % h, j = i + h;
        const double di = d[i], dj = d[j];
        double* col = a + (size_t)c * ld * ES;
#pragma unroll
        for (int part = 0; part < ES; ++part) {
            const double u = col[(size_t)i * ES + part], v = col[(size_t)j * ES + part];
            double x, y;
            if (kind == 0) {
                x = mul_rn(mul_rn(di, add_rn(u, v)), kInvSqrt2);
                y = mul_rn(mul_rn(dj, sub_rn(u, v)), kInvSqrt2);
            } else {
                const double p = mul_rn(di, u), r = mul_rn(dj, v);
                x = mul_rn(add_rn(p, r), kInvSqrt2);
                y = mul_rn(sub_rn(p, r), kInvSqrt2);
            }
            col[(size_t)i * ES + part] = x;
            col[(size_t)j * ES + part] = y;
        }
    }
}

// One butterfly level on the columns of a rows x N matrix: A := A B, the
// pairs (c, c + h) of every segment of 2h columns,
// (u, v) -> (d_c (u + v), d_{c+h} (u - v)) / sqrt 2 along each row.
template <bool CPLX>
__global__ void butterfly_cols_kernel(double* a, int ld, int rows, int n, int h, const double* d) {
    constexpr int ES = CPLX ? 2 : 1;
    const size_t total = (size_t)rows * (n / 2);
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(e % rows), q = (int)(e / rows);
        const int c = (q / h) * 2 * h + q % h, c2 = c + h;
        const double dc = d[c], dc2 = d[c2];
        double* pu = a + ((size_t)c * ld + r) * ES;
        double* pv = a + ((size_t)c2 * ld + r) * ES;
#pragma unroll
        for (int part = 0; part < ES; ++part) {
            const double u = pu[part], v = pv[part];
            pu[part] = mul_rn(mul_rn(dc, add_rn(u, v)), kInvSqrt2);
            pv[part] = mul_rn(mul_rn(dc2, sub_rn(u, v)), kInvSqrt2);
        }
    }
}

__global__ void unit_diagonal_kernel(double* a, int ld, int from, int to, int es) {
    const int i = from + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < to) a[((size_t)i * ld + i) * es] = 1.0;
}

// s[c * kNopivLd + r] := the rows x cols block at src (leading dimension ld),
// upper: zeros below the diagonal. Eight loads in flight per thread before
// their stores.
template <bool CPLX>
__device__ __forceinline__ void stage_block(Z* s, const double* src, int ld, int rows, int cols, bool upper) {
    constexpr int ES = CPLX ? 2 : 1;
    const int total = rows * cols;
    for (int e0 = threadIdx.x; e0 < total; e0 += 8 * blockDim.x) {
        Z v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * blockDim.x;
            v[u] = Z{0.0, 0.0};
            if (e < total) {
                const int r = e % rows, c = e / rows;
                if (!upper || r <= c) v[u] = load_el<CPLX>(src + ((size_t)c * ld + r) * ES);
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u * blockDim.x;
            if (e < total) s[(e / rows) * kNopivLd + e % rows] = v[u];
        }
    }
}

// The w x w diagonal block (w <= 64) factored in place without pivoting,
// L unit lower and U upper; an exactly zero pivot records its column (atomic
// minimum into flag) and the factorization goes on in inf/NaN.
template <bool CPLX>
__global__ void __launch_bounds__(256) lu_nopiv_diag_kernel(double* a, int ld, int w, int col0, int* flag) {
    constexpr int ES = CPLX ? 2 : 1;
    extern __shared__ __align__(16) unsigned char nopiv_smem[];
    Z* s = reinterpret_cast<Z*>(nopiv_smem);  // s[c * kNopivLd + r]
    stage_block<CPLX>(s, a, ld, w, w, false);
    __syncthreads();
    for (int k = 0; k < w; ++k) {
        const Z piv = s[k * kNopivLd + k];
        if (threadIdx.x == 0 && piv.re == 0.0 && piv.im == 0.0) atomicMin(flag, col0 + k);
        for (int r = k + 1 + threadIdx.x; r < w; r += blockDim.x)
            s[k * kNopivLd + r] = div_el<CPLX>(s[k * kNopivLd + r], piv);
        __syncthreads();
        const int m = w - k - 1;
        for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
            const int r = k + 1 + e % m, c = k + 1 + e / m;
            s[c * kNopivLd + r] = sub_prod<CPLX>(s[c * kNopivLd + r], s[k * kNopivLd + r], s[c * kNopivLd + k]);
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        const int r = e % w, c = e / w;
        store_el<CPLX>(a + ((size_t)c * ld + r) * ES, s[c * kNopivLd + r]);
    }
}

// X := X U^-1 for the rows x w block X (w <= 64) and the w x w upper factor
// U (staged in shared memory): one warp per row, lane l holding columns l and
// l + 32; step k divides x_k by u_kk in its lane, broadcasts it, and the lanes
// of the columns beyond k subtract x_k u_kc.
template <bool CPLX>
__global__ void __launch_bounds__(256) trsm_right_upper_kernel(const double* u, int ldu, double* x, int ldx,
                                                             int rows, int w) {
    constexpr int ES = CPLX ? 2 : 1;
    extern __shared__ __align__(16) unsigned char nopiv_smem[];
    Z* su = reinterpret_cast<Z*>(nopiv_smem);  // su[c * kNopivLd + r]
    stage_block<CPLX>(su, u, ldu, w, w, true);
    __syncthreads();
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int row = blockIdx.x * warps + (threadIdx.x >> 5); row < rows; row += gridDim.x * warps) {
        Z v[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int c = lane + 32 * q;
            v[q] = c < w ? load_el<CPLX>(x + ((size_t)c * ldx + row) * ES) : Z{0.0, 0.0};
        }
        for (int k = 0; k < w; ++k) {
            const int h = k >> 5, src = k & 31;
            if (lane == src) v[h] = div_el<CPLX>(v[h], su[k * kNopivLd + k]);
            const Z xk{__shfl_sync(0xffffffffu, v[h].re, src), CPLX ? __shfl_sync(0xffffffffu, v[h].im, src) : 0.0};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int c = lane + 32 * q;
                if (c > k && c < w) v[q] = sub_prod<CPLX>(v[q], xk, su[c * kNopivLd + k]);
            }
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int c = lane + 32 * q;
            if (c < w) store_el<CPLX>(x + ((size_t)c * ldx + row) * ES, v[q]);
        }
    }
}

constexpr int kNopivDiagSmem = kNopivBlock * kNopivLd * 16;
constexpr int kNopivTrsmSmem = kNopivBlock * kNopivLd * 16;

template <bool CPLX>
void configure_nopiv_kernels() {
    static bool done[64] = {};
    int dev = 0;
    TNS_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && done[dev]) return;
    TNS_CUDA(cudaFuncSetAttribute(lu_nopiv_diag_kernel<CPLX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kNopivDiagSmem));
    TNS_CUDA(cudaFuncSetAttribute(trsm_right_upper_kernel<CPLX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kNopivTrsmSmem));
    if (dev >= 0 && dev < 64) done[dev] = true;
}

// Inverses of the 64 x 64 diagonal blocks of packed factors without
// interchanges (n x n, unit lower L and upper U): one CTA per block, thread j
// of the first 64 computing column j of L_bb^-1 by forward substitution, of
// the next 64 column j of U_bb^-1 by back substitution. A partial last block
// is completed by the identity. inv holds nb blocks of L^-1, then nb of U^-1,
// each column-major with leading dimension 64.
template <bool CPLX>
__global__ void __launch_bounds__(128) diag_block_inverse_kernel(const double* f, int ld, int n, int nb,
                                                                double* inv) {
    constexpr int ES = CPLX ? 2 : 1;
    extern __shared__ __align__(16) unsigned char inv_smem[];
    Z* sd = reinterpret_cast<Z*>(inv_smem);  // the block, sd[c * kNopivLd + r]
    Z* sl = sd + kNopivBlock * kNopivLd;     // columns of L^-1
    Z* su = sl + kNopivBlock * kNopivLd;     // columns of U^-1
    const int b = blockIdx.x, r0 = b * kNopivBlock, w = min(kNopivBlock, n - r0);
    for (int e = threadIdx.x; e < kNopivBlock * kNopivBlock; e += blockDim.x) {
        const int r = e & 63, c = e >> 6;
        Z v = r == c ? Z{1.0, 0.0} : Z{0.0, 0.0};
        if (r < w && c < w) v = load_el<CPLX>(f + ((size_t)(r0 + c) * ld + r0 + r) * ES);
        sd[c * kNopivLd + r] = v;
    }
    __syncthreads();
    const int j = threadIdx.x & 63;
    if (threadIdx.x < 64) {
        Z* col = sl + j * kNopivLd;
        for (int i = 0; i < j; ++i) col[i] = Z{0.0, 0.0};
        col[j] = Z{1.0, 0.0};
        for (int i = j + 1; i < kNopivBlock; ++i) {
            Z acc{0.0, 0.0};
            for (int k = j; k < i; ++k) acc = sub_prod<CPLX>(acc, sd[k * kNopivLd + i], col[k]);
            col[i] = acc;
        }
    } else {
        Z* col = su + j * kNopivLd;
        for (int i = kNopivBlock - 1; i > j; --i) col[i] = Z{0.0, 0.0};
        for (int i = j; i >= 0; --i) {
            Z acc = i == j ? Z{1.0, 0.0} : Z{0.0, 0.0};
            for (int k = i + 1; k <= j; ++k) acc = sub_prod<CPLX>(acc, sd[k * kNopivLd + i], col[k]);
            col[i] = div_el<CPLX>(acc, sd[i * kNopivLd + i]);
        }
    }
    __syncthreads();
    double* il = inv + (size_t)b * kNopivBlock * kNopivBlock * ES;
    double* iu = inv + ((size_t)nb + b) * kNopivBlock * kNopivBlock * ES;
    for (int e = threadIdx.x; e < kNopivBlock * kNopivBlock; e += blockDim.x) {
        const int r = e & 63, c = e >> 6;
        store_el<CPLX>(il + (size_t)e * ES, sl[c * kNopivLd + r]);
        store_el<CPLX>(iu + (size_t)e * ES, su[c * kNopivLd + r]);
    }
}

__device__ __forceinline__ int ld_acquire_int(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_int(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
template <bool CPLX>
__device__ __forceinline__ Z load_el_cg(const double* p) {
    return CPLX ? Z{__ldcg(p), __ldcg(p + 1)} : Z{__ldcg(p), 0.0};
}

// Wait until block j of a chained solve is published; false (the error flag
// set) after kWaitTimeoutNs without it, or when another CTA gave up.
__device__ bool chain_wait(const int* flag, int* err) {
    if (ld_acquire_int(flag) != 0) return true;
    const unsigned long long start = global_timer_ns();
    for (unsigned it = 1;; ++it) {
        if (ld_acquire_int(flag) != 0) return true;
        if (it > 32) __nanosleep(64);
        if ((it & 255u) == 0) {
            if (*reinterpret_cast<volatile int*>(err) != 0) return false;
            if (global_timer_ns() - start > kWaitTimeoutNs) {
                atomicCAS(err, 0, kDevTimeoutChain);
                return false;
            }
        }
    }
}

constexpr int kChainCols = 4;  // right-hand sides per chained launch

// One triangle of packed factors without interchanges (n x n) applied as
// x := T^-1 x for up to 4 columns, row blocks of 64 chained through flags:
// the CTA owning block b subtracts T_bj x_j for every earlier block j as
// each is published, then x_b := T_bb^-1 (that sum) with the precomputed
// inverse, and publishes it. LOWERF: the unit lower factor L (else U); ADJ:
// T is the factor's conjugate transpose. Blocks go to CTAs in solve order and
// the launch is cooperative, so every block a CTA waits for is owned by a
// resident CTA that is working through earlier blocks only.
template <bool CPLX, bool LOWERF, bool ADJ>
__global__ void __launch_bounds__(256) chain_solve_kernel(const double* f, int ld, const double* inv, int n, int nb,
                                                        double* x, int ldx, int ncols, int* ready, int* err) {
    constexpr int ES = CPLX ? 2 : 1;
    constexpr bool FORWARD = LOWERF != ADJ;
    extern __shared__ __align__(16) unsigned char chain_smem[];
    Z* st = reinterpret_cast<Z*>(chain_smem);  // a 64 x 64 block, st[c * kNopivLd + r]
    Z* sx = st + kNopivBlock * kNopivLd;       // sx[c * 64 + k]
    __shared__ int s_ok;
    const int r = threadIdx.x & 63, c = threadIdx.x >> 6;
    const double* invs = inv + (LOWERF ? 0 : (size_t)nb * kNopivBlock * kNopivBlock * ES);
    for (int q = blockIdx.x; q < nb; q += gridDim.x) {
        const int b = FORWARD ? q : nb - 1 - q, r0 = b * kNopivBlock;
        Z acc = c < ncols ? load_el<CPLX>(x + ((size_t)c * ldx + r0 + r) * ES) : Z{0.0, 0.0};
        const int deps = FORWARD ? b : nb - 1 - b;
        for (int s = 0; s < deps; ++s) {
            const int j = FORWARD ? s : nb - 1 - s, j0 = j * kNopivBlock;
            __syncthreads();
            // T_bj: F[r0.., j0..] or, for the adjoint, conj(F[j0.., r0..])^T
            const int fr = ADJ ? j0 : r0, fc = ADJ ? r0 : j0;
            stage_block<CPLX>(st, f + ((size_t)fc * ld + fr) * ES, ld, kNopivBlock, kNopivBlock, false);
            if (threadIdx.x == 0) s_ok = chain_wait(ready + j, err) ? 1 : 0;
            __syncthreads();
            if (!s_ok) return;
            for (int e = threadIdx.x; e < kNopivBlock * ncols; e += blockDim.x) {
                const int k = e & 63, cc = e >> 6;
                sx[cc * kNopivBlock + k] = load_el_cg<CPLX>(x + ((size_t)cc * ldx + j0 + k) * ES);
            }
            __syncthreads();
            if (c < ncols) {
#pragma unroll 8
                for (int k = 0; k < kNopivBlock; ++k) {
                    Z t = ADJ ? st[r * kNopivLd + k] : st[k * kNopivLd + r];
                    if (ADJ) t.im = -t.im;
                    acc = sub_prod<CPLX>(acc, t, sx[c * kNopivBlock + k]);
                }
            }
        }
        __syncthreads();
        const double* ib = invs + (size_t)b * kNopivBlock * kNopivBlock * ES;
        stage_block<CPLX>(st, ib, kNopivBlock, kNopivBlock, kNopivBlock, false);
        if (c < ncols) sx[c * kNopivBlock + r] = acc;
        __syncthreads();
        if (c < ncols) {
            Z v{0.0, 0.0};
#pragma unroll 8
            for (int k = 0; k < kNopivBlock; ++k) {
                Z t = ADJ ? st[r * kNopivLd + k] : st[k * kNopivLd + r];
                if (ADJ) t.im = -t.im;
                v = sub_prod<CPLX>(v, Z{-t.re, -t.im}, sx[c * kNopivBlock + k]);
            }
            if (r0 + r < n) store_el<CPLX>(x + ((size_t)c * ldx + r0 + r) * ES, v);
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) st_release_int(ready + b, 1);
    }
}

constexpr int kInverseSmem = 3 * kNopivBlock * kNopivLd * 16;
constexpr int kChainSmem = kNopivBlock * kNopivLd * 16 + kChainCols * kNopivBlock * 16;

template <bool CPLX, bool LOWERF, bool ADJ>
void launch_chain(Context& ctx, const DMat& f, const double* inv, double* x, int ldx, int ncols, int* ready) {
    auto kernel = chain_solve_kernel<CPLX, LOWERF, ADJ>;
    static bool configured[64] = {};
    static int per_sm[64] = {};
    const int dev = ctx.device >= 0 && ctx.device < 64 ? ctx.device : 0;
    if (!configured[dev]) {
        TNS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kChainSmem));
        TNS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[dev], kernel, 256, kChainSmem));
        configured[dev] = true;
    }
    if (per_sm[dev] < 1) fail(TNS_E_DEVICE, "the chained triangular solve cannot be resident");
    const int n = f.rows, nb = (n + kNopivBlock - 1) / kNopivBlock;
    const int grid = std::min(nb, per_sm[dev] * ctx.num_sms);
    TNS_CUDA(cudaMemsetAsync(ready, 0, sizeof(int) * nb, ctx.stream));
    const double* fp = f.p;
    int ld = f.ld();
    int* err = ctx.d_err;
    void* args[] = {(void*)&fp, (void*)&ld, (void*)&inv, (void*)&n, (void*)&nb, (void*)&x, (void*)&ldx,
                    (void*)&ncols, (void*)&ready, (void*)&err};
    TNS_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kernel), dim3(grid), dim3(256), args, kChainSmem,
                                         ctx.stream));
    ctx.kernel_launches++;
}

// inv := the diagonal blocks' inverses of f (2 nb blocks of 64 x 64).
void diagonal_block_inverses(Context& ctx, const DMat& f, DBuf& inv) {
    const int n = f.rows, nb = (n + kNopivBlock - 1) / kNopivBlock;
    const size_t doubles = (size_t)2 * nb * kNopivBlock * kNopivBlock * (f.cplx ? 2 : 1);
    if (inv.bytes < sizeof(double) * doubles) inv = DBuf(ctx, sizeof(double) * doubles);
    static bool configured[2][64] = {};
    const int dev = ctx.device >= 0 && ctx.device < 64 ? ctx.device : 0;
    if (!configured[f.cplx][dev]) {
        if (f.cplx)
            TNS_CUDA(cudaFuncSetAttribute(diag_block_inverse_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kInverseSmem));
        else
            TNS_CUDA(cudaFuncSetAttribute(diag_block_inverse_kernel<false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, kInverseSmem));
        configured[f.cplx][dev] = true;
    }
    if (f.cplx)
        diag_block_inverse_kernel<true><<<nb, 128, kInverseSmem, ctx.stream>>>(f.p, f.ld(), n, nb, inv.as<double>());
    else
        diag_block_inverse_kernel<false><<<nb, 128, kInverseSmem, ctx.stream>>>(f.p, f.ld(), n, nb, inv.as<double>());
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

// x := (LU)^-1 x or (LU)^-H x for packed factors without interchanges, a few
// columns at a time through the chained kernel (the estimator's probes).
void chain_solve(Context& ctx, const DMat& f, const double* inv, DMat& x, int cols, bool adjoint) {
    const int nb = (f.rows + kNopivBlock - 1) / kNopivBlock;
    DBuf ready(ctx, sizeof(int) * nb);
    const size_t es = f.cplx ? 2 : 1;
    for (int c0 = 0; c0 < cols; c0 += kChainCols) {
        const int nc = std::min(kChainCols, cols - c0);
        double* xc = x.p + (size_t)c0 * x.ld() * es;
        if (f.cplx) {
            if (!adjoint) {
                launch_chain<true, true, false>(ctx, f, inv, xc, x.ld(), nc, ready.as<int>());
                launch_chain<true, false, false>(ctx, f, inv, xc, x.ld(), nc, ready.as<int>());
            } else {
                launch_chain<true, false, true>(ctx, f, inv, xc, x.ld(), nc, ready.as<int>());
                launch_chain<true, true, true>(ctx, f, inv, xc, x.ld(), nc, ready.as<int>());
            }
        } else {
            if (!adjoint) {
                launch_chain<false, true, false>(ctx, f, inv, xc, x.ld(), nc, ready.as<int>());
                launch_chain<false, false, false>(ctx, f, inv, xc, x.ld(), nc, ready.as<int>());
            } else {
                launch_chain<false, false, true>(ctx, f, inv, xc, x.ld(), nc, ready.as<int>());
                launch_chain<false, true, true>(ctx, f, inv, xc, x.ld(), nc, ready.as<int>());
            }
        }
    }
}

// Columns [j, j + w) of rows [j, n) factored without pivoting in 64-column
// steps: the diagonal block, L21 := A21 U11^-1, U12 := L11^-1 A12 within the
// panel, and the DMMA update of the panel's rest.
void lu_nopiv_panel(Context& ctx, DMat& a, int j, int w, int* flag) {
    const int n = a.rows, ld = a.ld();
    const bool cplx = a.cplx;
    if (cplx) configure_nopiv_kernels<true>();
    else configure_nopiv_kernels<false>();
    for (int b0 = 0; b0 < w; b0 += kNopivBlock) {
        const int bw = std::min(kNopivBlock, w - b0), k = j + b0;
        if (cplx) lu_nopiv_diag_kernel<true><<<1, 256, kNopivDiagSmem, ctx.stream>>>(a.at(k, k), ld, bw, k, flag);
        else lu_nopiv_diag_kernel<false><<<1, 256, kNopivDiagSmem, ctx.stream>>>(a.at(k, k), ld, bw, k, flag);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
        const int below = n - k - bw, right = w - b0 - bw;
        if (below > 0) {
            const int grid = std::min((below + 7) / 8, ctx.num_sms * 2);
            if (cplx)
                trsm_right_upper_kernel<true><<<grid, 256, kNopivTrsmSmem, ctx.stream>>>(a.at(k, k), ld,
                                                                                        a.at(k + bw, k), ld, below, bw);
            else
                trsm_right_upper_kernel<false><<<grid, 256, kNopivTrsmSmem, ctx.stream>>>(a.at(k, k), ld,
                                                                                         a.at(k + bw, k), ld, below, bw);
            TNS_CUDA(cudaGetLastError());
            ctx.kernel_launches++;
        }
        if (right > 0) {
            std::vector<TrsmDesc> t{TrsmDesc{a.at(k, k), ld, a.at(k, k + bw), ld, bw, right, 1, 1, 0}};
            launch_trsm(ctx, cplx, 1, t);
            if (below > 0) {
                GemmProblem p{};
                p.A = a.at(k + bw, k);
                p.B = a.at(k, k + bw);
                p.C = a.at(k + bw, k + bw);
                p.lda = p.ldb = p.ldc = ld;
                p.M = round_up(below, 2);
                p.N = round_up(right, 2);
                p.K = round_up(bw, 16);
                p.alpha_re = -1.0;
                p.beta_re = 1.0;
                p.work = (long long)below * right * bw;
                std::vector<GemmProblem> g{p};
                gemm_grouped(ctx, g, cplx);
            }
        }
    }
}

// The butterfly route; false (nothing of x written) when the elimination met
// an exactly zero pivot or the refinement did not reach an FP64 backward error.
bool gesv_mixed_butterfly(Context& ctx, const DMat& a, const DMat& b, DMat& x, int moduli, int max_iter,
                          MixedInfo& info) {
    const int n = a.rows, nrhs = b.cols;
    const bool cplx = a.cplx;
    const int es = cplx ? 2 : 1;
    const size_t esz = sizeof(double) * es;
    const int N = round_up(n, 4);
    info = MixedInfo{};

    // The four random diagonals (T1, T2, S1, S2), from a fixed seed.
    std::vector<double> dh(4 * (size_t)N);
    uint64_t state = 0x5DEECE66D2026ull;
    for (auto& v : dh) {
        state += 0x9E3779B97F4A7C15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const double r = (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
        v = std::exp(r / 10.0);
    }
    DBuf diag(ctx, sizeof(double) * dh.size());
    TNS_CUDA(cudaMemcpyAsync(diag.p, dh.data(), sizeof(double) * dh.size(), cudaMemcpyHostToDevice, ctx.stream));
    const double* dT1 = diag.as<double>();
    const double* dT2 = dT1 + N;
    const double* dS1 = dT1 + 2 * (size_t)N;
    const double* dS2 = dT1 + 3 * (size_t)N;
    const int grid = ctx.num_sms * 8;
    auto rows_level = [&](DMat& m, int cols, int h, const double* d, int kind) {
        if (cplx) butterfly_rows_kernel<true><<<grid, 256, 0, ctx.stream>>>(m.p, m.ld(), N, cols, h, d, kind);
        else butterfly_rows_kernel<false><<<grid, 256, 0, ctx.stream>>>(m.p, m.ld(), N, cols, h, d, kind);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
    };
    auto cols_level = [&](DMat& m, int h, const double* d) {
        if (cplx) butterfly_cols_kernel<true><<<grid, 256, 0, ctx.stream>>>(m.p, m.ld(), N, N, h, d);
        else butterfly_cols_kernel<false><<<grid, 256, 0, ctx.stream>>>(m.p, m.ld(), N, N, h, d);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
    };

    // T A S, A embedded as [[A, 0], [0, I]].
    DMat t(ctx, N, N, cplx, "the transformed matrix of a butterfly solve");
    TNS_CUDA(cudaMemcpy2DAsync(t.p, (size_t)t.ld() * esz, a.p, (size_t)a.ld() * esz, (size_t)n * esz, n,
                               cudaMemcpyDeviceToDevice, ctx.stream));
    if (N > n) {
        unit_diagonal_kernel<<<1, 32, 0, ctx.stream>>>(t.p, t.ld(), n, N, es);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
    }
    rows_level(t, N, N / 2, dT1, 0);
    rows_level(t, N, N / 4, dT2, 0);
    cols_level(t, N / 2, dS1);
    cols_level(t, N / 4, dS2);

    DMat f(ctx, N, N, cplx, "the low-precision factors");
    DBuf flag(ctx, sizeof(int));
    DBuf inverses;  // the factors' diagonal blocks, inverted, for the chained solves
    auto factor = [&](int m) {
        copy_dmat(ctx, f, t);
        const int init = INT_MAX;
        TNS_CUDA(cudaMemcpyAsync(flag.p, &init, sizeof(int), cudaMemcpyHostToDevice, ctx.stream));
        for (int j = 0; j < N; j += kMixedOuter) {
            const int w = std::min(kMixedOuter, N - j);
            lu_nopiv_panel(ctx, f, j, w, flag.as<int>());
            if (j + w < N) mixed_trailing(ctx, f, j, w, m);
        }
        diagonal_block_inverses(ctx, f, inverses);
        int zero_at = INT_MAX;
        TNS_CUDA(cudaMemcpyAsync(&zero_at, flag.p, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        info.factorizations++;
        info.moduli = m;
        return zero_at == INT_MAX;
    };
    // (LU)^-1 or (LU)^-H in place: a few columns (the estimator's probes)
    // through the chained solve, wide panels by blocked TRSM + DMMA updates.
    auto lu_solve = [&](DMat& m, int cols, bool adjoint) {
        if (cols <= 2 * kChainCols) chain_solve(ctx, f, inverses.as<double>(), m, cols, adjoint);
        else getrs_free_order(ctx, f, nullptr, m, cols, adjoint);
    };
    // M := A^-1 M or A^-H M in place on an N-row panel (zeros below row n).
    const std::function<void(DMat&, int, bool)> solve = [&](DMat& m, int cols, bool adjoint) {
        if (!adjoint) {
            rows_level(m, cols, N / 2, dT1, 0);
            rows_level(m, cols, N / 4, dT2, 0);
            lu_solve(m, cols, false);
            rows_level(m, cols, N / 4, dS2, 1);
            rows_level(m, cols, N / 2, dS1, 1);
        } else {
            rows_level(m, cols, N / 2, dS1, 0);
            rows_level(m, cols, N / 4, dS2, 0);
            lu_solve(m, cols, true);
            rows_level(m, cols, N / 4, dT2, 1);
            rows_level(m, cols, N / 2, dT1, 1);
        }
    };

    if (!factor(moduli > 0 ? moduli : 8)) return false;
    const double anorm1 = norm1(ctx, a);
    const NormestResult est = normest_solve(ctx, n, N, cplx, solve, 2, 5, 20260915);
    info.rcond = (anorm1 > 0.0 && est.value > 0.0) ? 1.0 / (anorm1 * est.value) : 0.0;
    if (!std::isfinite(est.value)) return false;
    if (moduli == 0) {
        // Without pivoting the factors may grow (small pivots are rare but not
        // excluded): the images keep log2(kappa_1) + log2(growth) + 7 bits,
        // growth = max |L\U| / max |T A S|.
        auto absmax = [&](const DMat& m) {
            const std::vector<double> c = col_absmax(ctx, m);
            return c.empty() ? 0.0 : *std::max_element(c.begin(), c.end());
        };
        const double fmax = absmax(f), tmax = absmax(t);
        if (!std::isfinite(fmax)) return false;
        const double growth = tmax > 0.0 ? std::max(1.0, fmax / tmax) : 1.0;
        const double kappa = info.rcond > 0.0 ? 1.0 / info.rcond : 1e300;
        const int need = (int)std::ceil(std::log2(std::max(1.0, kappa)) + std::log2(growth)) + 7;
        const int depth = cplx ? 2 * kMixedOuter : kMixedOuter;
        int m = info.moduli;
        while (m < 22 && split_integer_bits(m, depth) < need) ++m;
        if (m > info.moduli) {
            if (!factor(m)) return false;
            // The first factors may have inflated the estimate: take it again
            // from the factors the refinement uses.
            const NormestResult again = normest_solve(ctx, n, N, cplx, solve, 2, 5, 20260915);
            if (!std::isfinite(again.value)) return false;
            info.rcond = (anorm1 > 0.0 && again.value > 0.0) ? 1.0 / (anorm1 * again.value) : 0.0;
        }
    }

    // x on N rows; the residual's rows below n stay zero.
    DMat xs(ctx, N, nrhs, cplx, "the solution");
    TNS_CUDA(cudaMemcpy2DAsync(xs.p, (size_t)xs.ld() * esz, b.p, (size_t)b.ld() * esz, (size_t)n * esz, nrhs,
                               cudaMemcpyDeviceToDevice, ctx.stream));
    solve(xs, nrhs, false);
    DMat xv = block_view(xs, 0, 0, n, nrhs);
    DMat r(ctx, N, nrhs, cplx, "the refinement residual");
    DMat rv = block_view(r, 0, 0, n, nrhs);
    const double ainf = norminf(ctx, a);
    const std::vector<double> bmax = col_absmax(ctx, b);
    double prev = INFINITY;
    for (int it = 0;; ++it) {
        TNS_CUDA(cudaMemcpy2DAsync(r.p, (size_t)r.ld() * esz, b.p, (size_t)b.ld() * esz, (size_t)n * esz, nrhs,
                                   cudaMemcpyDeviceToDevice, ctx.stream));
        std::vector<GemmProblem> g{make_gemm(a, xv, rv, -1.0, 0.0, 1.0, 0.0)};
        gemm_grouped(ctx, g, cplx);
        const std::vector<double> rmax = col_absmax(ctx, rv), xmax = col_absmax(ctx, xv);
        double berr = 0.0;
        for (int j = 0; j < nrhs; ++j) {
            const double den = ainf * xmax[j] + bmax[j];
            berr = std::max(berr, den > 0.0 ? rmax[j] / den : (rmax[j] > 0.0 ? INFINITY : 0.0));
        }
        info.backward_error = berr;
        if (berr <= 4.0 * 1.1102230246251565e-16 || it >= max_iter || !(berr < 0.5 * prev)) break;
        prev = berr;
        solve(r, nrhs, false);
        std::vector<EwDesc> add{ew_add_scaled(xs, r, 1.0)};
        ew_batch(ctx, add);
        info.iterations++;
    }
    // An FP64 backward error (8 u), or the pivoting route decides.
    if (!(info.backward_error <= 8.0 * 1.1102230246251565e-16)) return false;
    x = DMat(ctx, n, nrhs, cplx, "the solution");
    TNS_CUDA(cudaMemcpy2DAsync(x.p, (size_t)x.ld() * esz, xs.p, (size_t)xs.ld() * esz, (size_t)n * esz, nrhs,
                               cudaMemcpyDeviceToDevice, ctx.stream));
    return true;
}

}  // namespace

void gesv_mixed(Context& ctx, const DMat& a, const DMat& b, DMat& x, int moduli, int max_iter, MixedInfo& info) {
    if (gesv_mixed_butterfly(ctx, a, b, x, moduli, max_iter, info)) return;
    const int tried = info.factorizations;
    gesv_mixed_pivoted(ctx, a, b, x, moduli, max_iter, info);
    info.factorizations += tried;
}

}  // namespace tns
