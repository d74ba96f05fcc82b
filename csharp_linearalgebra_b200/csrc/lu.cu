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
// solve included -- matches the reference bit for bit. The adjoint solves use
// 64-row diagonal blocks plus DMMA GEMM updates of the rows beyond them (a
// blocked, GEMM-based TRSM).

#include "batch.cuh"
#include "device_util.cuh"
#include "tns_internal.h"

#include <algorithm>
#include <climits>
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
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        int i = e % w, p = e / w;
        int si = d.conj ? p : i, sp = d.conj ? i : p;
        const double* src = d.t + ((size_t)sp * d.ldt + si) * ES;
        sT[(size_t)e * ES] = src[0];
        if (CPLX) sT[(size_t)e * ES + 1] = d.conj ? -src[1] : src[1];
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
template <bool CPLX, bool UPPER>
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
        for (int k = 0; k < B - 1; ++k) {
            const Z xk = v[k];
            if (k >= w || (xk.re == 0.0 && xk.im == 0.0)) continue;
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

// Step 2: rows [r0, r1) of every column take the updates of steps [k0, k1)
// (ascending for the lower factor, descending for the upper), 64 x 64 tiles
// of (row, column) per CTA over a flat grid of every item's tiles. Thread
// (tx, ty) keeps rows tx + 16 r and columns ty + 16 s (r, s < 4) in registers
// from the value x already holds; each round stages 16 steps of the factor
// column and of the solved x[k] in shared memory.
template <bool CPLX, bool UPPER>
__global__ void __launch_bounds__(256, 2) subst_update_kernel(const __grid_constant__ Batch<SubstUpdateDesc> b) {
    constexpr int ES = CPLX ? 2 : 1;
    constexpr int KC = 16;
    int lo = 0, hi = b.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (batch_item(b, mid).tile_begin <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const SubstUpdateDesc& d = batch_item(b, lo);
    const int tile = blockIdx.x - d.tile_begin;
    const int i0 = d.r0 + (tile % d.tiles_m) * 64, c0 = (tile / d.tiles_m) * 64;
    __shared__ Z sF[KC][64];
    __shared__ Z sX[KC][64 + 1];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
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
    const int rounds = (d.k1 - d.k0 + KC - 1) / KC;
    for (int q = 0; q < rounds; ++q) {
        const int kq = UPPER ? d.k1 - (q + 1) * KC : d.k0 + q * KC;
        for (int e = tid; e < KC * 64; e += 256) {
            const int kk = e >> 6, r = e & 63;
            const int k = kq + kk, i = i0 + r;
            Z v{0.0, 0.0};
            if (k >= d.k0 && k < d.k1 && i < d.r1) {
                const double* p = d.f + ((size_t)k * d.ldf + i) * ES;
                v = Z{p[0], CPLX ? p[1] : 0.0};
            }
            sF[kk][r] = v;
        }
        for (int e = tid; e < KC * 64; e += 256) {
            const int kk = e % KC, c = e / KC;
            const int k = kq + kk, col = c0 + c;
            Z v{0.0, 0.0};  // steps outside [k0, k1) read as zero and are skipped
            if (k >= d.k0 && k < d.k1 && col < d.nrhs) {
                const double* p = d.x + ((size_t)col * d.ldx + k) * ES;
                v = Z{p[0], CPLX ? p[1] : 0.0};
            }
            sX[kk][c] = v;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < KC; ++j) {
            const int kk = UPPER ? KC - 1 - j : j;
            Z nxk[4];
            bool live[4];
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const Z xv = sX[kk][ty + 16 * s];
                live[s] = !(xv.re == 0.0 && xv.im == 0.0);
                nxk[s] = Z{-xv.re, -xv.im};
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const Z fv = sF[kk][tx + 16 * r];
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

void launch_panels(Context& ctx, bool cplx, std::vector<PanelFactorDesc>& v) {
    if (v.empty()) return;
    Batch<PanelFactorDesc> b = make_batch(ctx, v);
    if (cplx) panel_kernel<true><<<b.count, 512, 0, ctx.stream>>>(b);
    else panel_kernel<false><<<b.count, 512, 0, ctx.stream>>>(b);
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
template <bool CPLX, bool UPPER>
void launch_subst_step_t(Context& ctx, std::vector<SubstDiagDesc>& diag, std::vector<SubstUpdateDesc>& upd) {
    if (!diag.empty()) {
        int mr = 0;
        for (auto& d : diag) mr = std::max(mr, d.nrhs);
        Batch<SubstDiagDesc> b = make_batch(ctx, diag);
        subst_diag_kernel<CPLX, UPPER><<<dim3((mr + 127) / 128, b.count), 128, 0, ctx.stream>>>(b);
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
        subst_update_kernel<CPLX, UPPER><<<(unsigned)total, 256, 0, ctx.stream>>>(b);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
    }
}

void launch_subst_step(Context& ctx, bool cplx, bool upper, std::vector<SubstDiagDesc>& diag,
                       std::vector<SubstUpdateDesc>& upd) {
    if (cplx) {
        if (upper) launch_subst_step_t<true, true>(ctx, diag, upd);
        else launch_subst_step_t<true, false>(ctx, diag, upd);
    } else {
        if (upper) launch_subst_step_t<false, true>(ctx, diag, upd);
        else launch_subst_step_t<false, false>(ctx, diag, upd);
    }
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
        launch_panels(ctx, cplx, panels);
        launch_laswp(ctx, cplx, swaps);
        launch_trsm(ctx, cplx, 0, trsms);
        if (!gemms.empty()) gemm_grouped(ctx, gemms, cplx);
    }
}

void getrs_batch(Context& ctx, std::vector<SolveItem>& items, bool adjoint) {
    if (items.empty()) return;
    const bool cplx = items[0].lu->cplx;
    const int bs = 64;
    const size_t es = cplx ? 2 : 1;
    int max_blocks = 0;
    std::vector<DMat> herm;  // conjugate transposes for the adjoint solves
    for (auto& it : items) {
        int n = it.lu->rows;
        if (n == 0 || it.nrhs == 0) continue;
        max_blocks = std::max(max_blocks, (n + bs - 1) / bs);
    }
    if (adjoint) {
        herm.reserve(items.size());
        for (auto& it : items) {
            herm.emplace_back(ctx, it.lu->cols, it.lu->rows, cplx, "the conjugate transpose of the factors");
            conj_transpose(ctx, herm.back(), *it.lu);
        }
    }
    auto update = [&](std::vector<GemmProblem>& v, const double* A, int lda, const double* X, double* C, int ldb,
                      int rows, int k, int nrhs) {
        if (rows <= 0) return;
        GemmProblem p{};
        p.A = A;
        p.B = X;
        p.C = C;
        p.lda = lda;
        p.ldb = p.ldc = ldb;
        p.M = round_up(rows, 2);
        p.N = round_up(nrhs, 2);
        p.K = round_up(k, 16);
        p.alpha_re = -1.0;
        p.beta_re = 1.0;
        v.push_back(p);
    };
    if (!adjoint) {
        // P B, then L (unit lower) forward and U backward by substitution in
        // the reference's order (Lu.Solve, Lu.cs:336-351; BlockedLu.Solve,
        // BlockedLu.cs:105-118): the result matches the reference bit for bit.
        std::vector<LaswpDesc> swaps;
        constexpr int B = kSubstBlock;
        int steps = 0;
        for (auto& it : items) {
            int n = it.lu->rows;
            if (n == 0 || it.nrhs == 0) continue;
            swaps.push_back(LaswpDesc{it.b->p, it.b->ld(), 0, it.nrhs, it.d_piv, 0, n, 0});
            steps = std::max(steps, (n + B - 1) / B);
        }
        launch_laswp(ctx, cplx, swaps);
        // Lower: blocks from the top; upper: each item's blocks from its last.
        for (int upper = 0; upper < 2; ++upper)
            for (int s = 0; s < steps; ++s) {
                std::vector<SubstDiagDesc> diag;
                std::vector<SubstUpdateDesc> upd;
                for (auto& it : items) {
                    const int n = it.lu->rows;
                    if (n == 0 || it.nrhs == 0) continue;
                    const int blocks = (n + B - 1) / B;
                    if (s >= blocks) continue;
                    const int k0 = (upper ? blocks - 1 - s : s) * B, w = std::min(B, n - k0);
                    const int ldf = it.lu->ld(), ldx = it.b->ld();
                    diag.push_back(SubstDiagDesc{it.lu->p, ldf, it.b->p, ldx, it.nrhs, k0, w});
                    const int r0 = upper ? 0 : k0 + w, r1 = upper ? k0 : n;
                    if (r1 > r0)
                        upd.push_back(SubstUpdateDesc{it.lu->p, ldf, it.b->p, ldx, it.nrhs, r0, r1, k0, k0 + w,
                                                      (r1 - r0 + 63) / 64, 0});
                }
                launch_subst_step(ctx, cplx, upper != 0, diag, upd);
            }
        return;
    }
    // The adjoint: blocked, 64-row diagonal blocks plus DMMA GEMM updates.
    // Pass 1: forward (U^H, non-unit).
    for (int kb = 0; kb < max_blocks; ++kb) {
        std::vector<TrsmDesc> diag;
        std::vector<GemmProblem> gemms;
        for (size_t q = 0; q < items.size(); ++q) {
            auto& it = items[q];
            const DMat& F = *it.lu;
            int n = F.rows, ld = F.ld(), ldb = it.b->ld();
            int k0 = kb * bs;
            if (n == 0 || it.nrhs == 0 || k0 >= n) continue;
            int w = std::min(bs, n - k0);
            double* B = it.b->p;
            diag.push_back(TrsmDesc{F.p + ((size_t)k0 * ld + k0) * es, ld, B + (size_t)k0 * es, ldb, w, it.nrhs, 1,
                                    adjoint ? 0 : 1, adjoint ? 1 : 0});
            const double* A = adjoint ? herm[q].p + ((size_t)k0 * herm[q].ld() + k0 + w) * es
                                      : F.p + ((size_t)k0 * ld + k0 + w) * es;
            update(gemms, A, adjoint ? herm[q].ld() : ld, B + (size_t)k0 * es, B + (size_t)(k0 + w) * es, ldb,
                   n - k0 - w, w, it.nrhs);
        }
        launch_trsm(ctx, cplx, 1, diag);
        if (!gemms.empty()) gemm_grouped(ctx, gemms, cplx);
    }
    // Pass 2: backward (U, non-unit; or L^H, unit, for the adjoint).
    for (int kb = max_blocks - 1; kb >= 0; --kb) {
        std::vector<TrsmDesc> diag;
        std::vector<GemmProblem> gemms;
        for (size_t q = 0; q < items.size(); ++q) {
            auto& it = items[q];
            const DMat& F = *it.lu;
            int n = F.rows, ld = F.ld(), ldb = it.b->ld();
            int k0 = kb * bs;
            if (n == 0 || it.nrhs == 0 || k0 >= n) continue;
            int w = std::min(bs, n - k0);
            double* B = it.b->p;
            diag.push_back(TrsmDesc{F.p + ((size_t)k0 * ld + k0) * es, ld, B + (size_t)k0 * es, ldb, w, it.nrhs, 0,
                                    adjoint ? 1 : 0, adjoint ? 1 : 0});
            const double* A = adjoint ? herm[q].p + ((size_t)k0 * herm[q].ld()) * es : F.p + ((size_t)k0 * ld) * es;
            update(gemms, A, adjoint ? herm[q].ld() : ld, B + (size_t)k0 * es, B, ldb, k0, w, it.nrhs);
        }
        launch_trsm(ctx, cplx, 1, diag);
        if (!gemms.empty()) gemm_grouped(ctx, gemms, cplx);
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

}  // namespace tns
