// LU with partial pivoting and the triangular solves, on the GPU.
//
// Right-looking blocked getrf as the reference runs it (src/Tensile.Kernels/Lu.cs:230-309
// for real, src/Tensile/BlockedLu.cs:45-101 for complex): per block of nb
// columns
//   1. panel factorization (one CTA; pivot = first index of the largest |a|,
//      or |Re|+|Im| for complex; reciprocal multiply unless |pivot| < SafeMin;
//      rank-1 updates y + (-m)*x with two roundings),
//   2. the panel's row interchanges applied to the columns either side,
//   3. U12 := L11^-1 A12 (one warp per column, the reference's update order),
//   4. A22 := A22 - A21*U12 on the DMMA GEMM.
// The per-element arithmetic of steps 1-3 is the reference's, so the pivot
// sequence can only differ from the reference through the trailing GEMM's
// summation order.
//
// Solves: few right-hand sides use one CTA per column (substitution with the
// reference's update order); many right-hand sides (the Pade solve, n RHS)
// use 64-row diagonal-block substitution plus DMMA GEMM updates, a blocked
// TRSM (the reference's own planned next step, GEMM-based TRSM).

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
// one CTA. pivots land as global 0-based rows in piv[r0 + j].
// ---------------------------------------------------------------------------
template <bool CPLX>
__global__ void __launch_bounds__(512) panel_kernel(double* a, int ld, int m, int r0, int w, int* piv, int* singular) {
    constexpr int ES = CPLX ? 2 : 1;
    __shared__ double s_val[32];
    __shared__ int s_idx[32];
    __shared__ int s_p;
    __shared__ double s_prow[2 * 64];
    const int tid = threadIdx.x;
    const int nthreads = blockDim.x;
    const int M = m - r0;  // rows in the panel
    const int limit = min(M, w);
    double* P = a + ((size_t)r0 * ld + r0) * ES;  // panel origin

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
            piv[r0 + j] = r0 + bi;
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
                if (tid == 0) atomicMin(singular, r0 + j);
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
            if (zero && tid == 0) atomicMin(singular, r0 + j);
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
// k, to columns [c0, c1). One thread per column (SwapRows, Lu.cs:430-448).
template <bool CPLX>
__global__ void laswp_kernel(double* a, int ld, int c0, int c1, const int* piv, int k0, int k1, bool reverse) {
    constexpr int ES = CPLX ? 2 : 1;
    int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c1) return;
    double* col = a + (size_t)c * ld * ES;
    for (int s = 0; s < k1 - k0; ++s) {
        int k = reverse ? k1 - 1 - s : k0 + s;
        int p = piv[k];
        if (p != k) {
            for (int q = 0; q < ES; ++q) {
                double tmp = col[(size_t)k * ES + q];
                col[(size_t)k * ES + q] = col[(size_t)p * ES + q];
                col[(size_t)p * ES + q] = tmp;
            }
        }
    }
}

// B := L^-1 B for a w x w unit lower L (w <= 64) at `l`, B w x ncols at `b`.
// One warp per column, x[i] += (-x[p]) * L[i, p] for p = 0..w-2 in order
// (Triangular.SolveLowerUnit, Triangular.cs:26-57; complex BlockedLu.cs:312-327).
template <bool CPLX>
__global__ void trsm_lower_unit_kernel(const double* l, int ldl, double* b, int ldb, int w, int ncols) {
    constexpr int ES = CPLX ? 2 : 1;
    extern __shared__ double sL[];  // w x w, ld w
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        int i = e % w, p = e / w;
        for (int q = 0; q < ES; ++q) sL[(size_t)e * ES + q] = l[((size_t)p * ldl + i) * ES + q];
    }
    __syncthreads();
    int lane = threadIdx.x & 31;
    int warps = blockDim.x >> 5;
    for (int c = blockIdx.x * warps + (threadIdx.x >> 5); c < ncols; c += gridDim.x * warps) {
        double* x = b + (size_t)c * ldb * ES;
        double xr[2], xi[2];
        for (int h = 0; h < 2; ++h) {
            int i = lane + 32 * h;
            xr[h] = i < w ? x[(size_t)i * ES] : 0.0;
            xi[h] = (CPLX && i < w) ? x[(size_t)i * ES + 1] : 0.0;
        }
        for (int p = 0; p < w - 1; ++p) {
            double vr = __shfl_sync(0xffffffffu, xr[p >> 5], p & 31);
            double vi = CPLX ? __shfl_sync(0xffffffffu, xi[p >> 5], p & 31) : 0.0;
            if (vr == 0.0 && vi == 0.0) continue;
            for (int h = 0; h < 2; ++h) {
                int i = lane + 32 * h;
                if (i > p && i < w) {
                    if (!CPLX) {
                        xr[h] = add_rn(xr[h], mul_rn(-vr, sL[(size_t)p * w + i]));
                    } else {
                        Z lv{sL[((size_t)p * w + i) * 2], sL[((size_t)p * w + i) * 2 + 1]};
                        Z r = zadd(Z{xr[h], xi[h]}, zmul(Z{-vr, -vi}, lv));
                        xr[h] = r.re;
                        xi[h] = r.im;
                    }
                }
            }
        }
        for (int h = 0; h < 2; ++h) {
            int i = lane + 32 * h;
            if (i < w) {
                x[(size_t)i * ES] = xr[h];
                if (CPLX) x[(size_t)i * ES + 1] = xi[h];
            }
        }
    }
}

// Diagonal-block substitution for the blocked solves: X := T^-1 X with T the
// w x w block (w <= 64) at `t`: lower or upper, unit or not, optionally the
// conjugate transpose of the stored block. One warp per right-hand side.
template <bool CPLX>
__global__ void trsm_block_kernel(const double* t, int ldt, double* b, int ldb, int w, int ncols, bool lower, bool unit,
                                  bool conj_trans) {
    constexpr int ES = CPLX ? 2 : 1;
    extern __shared__ double sT[];  // effective operator, w x w, ld w: op(i, p)
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        int i = e % w, p = e / w;
        // op(i, p) = stored(i, p), or conj(stored(p, i)) for the adjoint
        int si = conj_trans ? p : i, sp = conj_trans ? i : p;
        sT[(size_t)e * ES] = t[((size_t)sp * ldt + si) * ES];
        if (CPLX) sT[(size_t)e * ES + 1] = conj_trans ? -t[((size_t)sp * ldt + si) * ES + 1] : t[((size_t)sp * ldt + si) * ES + 1];
    }
    __syncthreads();
    int lane = threadIdx.x & 31;
    int warps = blockDim.x >> 5;
    for (int c = blockIdx.x * warps + (threadIdx.x >> 5); c < ncols; c += gridDim.x * warps) {
        double* x = b + (size_t)c * ldb * ES;
        Z v[2];
        for (int h = 0; h < 2; ++h) {
            int i = lane + 32 * h;
            v[h].re = i < w ? x[(size_t)i * ES] : 0.0;
            v[h].im = (CPLX && i < w) ? x[(size_t)i * ES + 1] : 0.0;
        }
        for (int s = 0; s < w; ++s) {
            int p = lower ? s : w - 1 - s;
            int h = p >> 5, src = p & 31;
            if (!unit) {
                if (lane == src) {
                    if (!CPLX) {
                        v[h].re = __ddiv_rn(v[h].re, sT[(size_t)p * w + p]);
                    } else {
                        Z d{sT[((size_t)p * w + p) * 2], sT[((size_t)p * w + p) * 2 + 1]};
                        v[h] = zdiv(v[h], d);
                    }
                }
            }
            double vr = __shfl_sync(0xffffffffu, v[h].re, src);
            double vi = CPLX ? __shfl_sync(0xffffffffu, v[h].im, src) : 0.0;
            for (int q = 0; q < 2; ++q) {
                int i = lane + 32 * q;
                bool below = lower ? (i > p) : (i < p);
                if (below && i < w) {
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

__global__ void init_int_kernel(int* p, int v) { *p = v; }

// The 64 x 64 complex block needs 64 KB of dynamic shared memory, above the
// default 48 KB, so the triangular kernels opt in before each launch (the
// attribute is per kernel; real and complex instances share a signature, so
// no static flag can tell them apart).
template <class K>
void allow_64k_smem(Context&, K kernel) {
    TNS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 64 * 16));
}

template <bool CPLX>
void launch_trsm_lower_unit(Context& ctx, const double* l, int ldl, double* b, int ldb, int w, int ncols) {
    if (ncols <= 0 || w <= 1) return;
    allow_64k_smem(ctx, trsm_lower_unit_kernel<CPLX>);
    int threads = 256;
    int warps = threads / 32;
    int grid = std::min((ncols + warps - 1) / warps, ctx.num_sms * 4);
    size_t smem = (size_t)w * w * (CPLX ? 16 : 8);
    trsm_lower_unit_kernel<CPLX><<<grid, threads, smem, ctx.stream>>>(l, ldl, b, ldb, w, ncols);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

template <bool CPLX>
void launch_trsm_block(Context& ctx, const double* t, int ldt, double* b, int ldb, int w, int ncols, bool lower, bool unit,
                       bool conj_trans) {
    if (ncols <= 0 || w <= 0) return;
    allow_64k_smem(ctx, trsm_block_kernel<CPLX>);
    int threads = 256;
    int warps = threads / 32;
    int grid = std::min((ncols + warps - 1) / warps, ctx.num_sms * 4);
    size_t smem = (size_t)w * w * (CPLX ? 16 : 8);
    trsm_block_kernel<CPLX><<<grid, threads, smem, ctx.stream>>>(t, ldt, b, ldb, w, ncols, lower, unit, conj_trans);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void launch_laswp(Context& ctx, bool cplx, double* a, int ld, int c0, int c1, const int* piv, int k0, int k1, bool reverse) {
    if (c1 <= c0 || k1 <= k0) return;
    int n = c1 - c0;
    if (cplx)
        laswp_kernel<true><<<(n + 127) / 128, 128, 0, ctx.stream>>>(a, ld, c0, c1, piv, k0, k1, reverse);
    else
        laswp_kernel<false><<<(n + 127) / 128, 128, 0, ctx.stream>>>(a, ld, c0, c1, piv, k0, k1, reverse);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

// Element offset (in doubles) of (i, j) in a padded matrix.
inline size_t off(const DMat& a, int i, int j) { return ((size_t)j * a.ld() + i) * (a.cplx ? 2 : 1); }

}  // namespace

LuResult getrf(Context& ctx, DMat& a, int m, int n, int nb, int* d_piv) {
    LuResult res;
    int limit = std::min(m, n);
    if (limit == 0) return res;
    if (nb < 1) nb = std::min(m, n) < 1024 ? 32 : 64;
    // The GEMM wants K % 16 == 0 and the panel's pivot row buffer holds 64.
    nb = std::max(16, std::min(64, (nb + 15) / 16 * 16));
    const bool cplx = a.cplx;
    const int ld = a.ld();
    DBuf flags(ctx, sizeof(int) + 2 * sizeof(double) + 8);
    int* d_sing = flags.as<int>();
    double* d_range = reinterpret_cast<double*>(flags.as<char>() + 8);
    init_int_kernel<<<1, 1, 0, ctx.stream>>>(d_sing, INT_MAX);
    ctx.kernel_launches++;

    auto panel = [&](int r0, int w) {
        if (cplx)
            panel_kernel<true><<<1, 512, 0, ctx.stream>>>(a.p, ld, m, r0, w, d_piv, d_sing);
        else
            panel_kernel<false><<<1, 512, 0, ctx.stream>>>(a.p, ld, m, r0, w, d_piv, d_sing);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
    };

    if (nb >= limit) {
        // Whole-matrix panel (Lu.cs:244-249): factor n columns at once is only
        // possible when n <= 64 (pivot-row buffer); wider unblocked shapes go
        // through the blocked path, which gives the same pivots.
        if (n <= 64) {
            panel(0, n);
        } else {
            panel(0, limit);
            launch_laswp(ctx, cplx, a.p, ld, limit, n, d_piv, 0, limit, false);
            if (cplx)
                launch_trsm_lower_unit<true>(ctx, a.p, ld, a.p + off(a, 0, limit), ld, limit, n - limit);
            else
                launch_trsm_lower_unit<false>(ctx, a.p, ld, a.p + off(a, 0, limit), ld, limit, n - limit);
        }
    } else {
        for (int jb = 0; jb < limit; jb += nb) {
            int w = std::min(nb, limit - jb);
            panel(jb, w);
            launch_laswp(ctx, cplx, a.p, ld, 0, jb, d_piv, jb, jb + w, false);
            if (jb + w >= n) continue;
            launch_laswp(ctx, cplx, a.p, ld, jb + w, n, d_piv, jb, jb + w, false);
            if (cplx)
                launch_trsm_lower_unit<true>(ctx, a.p + off(a, jb, jb), ld, a.p + off(a, jb, jb + w), ld, w, n - jb - w);
            else
                launch_trsm_lower_unit<false>(ctx, a.p + off(a, jb, jb), ld, a.p + off(a, jb, jb + w), ld, w, n - jb - w);
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
            gemm(ctx, p, cplx);
        }
    }
    if (cplx)
        pivot_range_kernel<true><<<1, 256, 0, ctx.stream>>>(a.p, ld, limit, d_range);
    else
        pivot_range_kernel<false><<<1, 256, 0, ctx.stream>>>(a.p, ld, limit, d_range);
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
    const int n = lu.rows;
    if (n == 0 || nrhs == 0) return;
    const bool cplx = lu.cplx;
    const int ld = lu.ld();
    const int ldb = b.ld();
    const int bs = 64;
    double* B = b.p;
    const double* F = lu.p;
    auto trsm = [&](const double* t, double* x, int w, bool lower, bool unit, bool ct) {
        if (cplx) launch_trsm_block<true>(ctx, t, ld, x, ldb, w, nrhs, lower, unit, ct);
        else launch_trsm_block<false>(ctx, t, ld, x, ldb, w, nrhs, lower, unit, ct);
    };
    auto update = [&](const double* A, int lda, const double* X, double* C, int rows, int k) {
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
        gemm(ctx, p, cplx);
    };
    const size_t es = cplx ? 2 : 1;
    if (!adjoint) {
        launch_laswp(ctx, cplx, B, ldb, 0, nrhs, d_piv, 0, n, false);
        // L (unit lower): forward, block by block.
        for (int k0 = 0; k0 < n; k0 += bs) {
            int w = std::min(bs, n - k0);
            trsm(F + ((size_t)k0 * ld + k0) * es, B + (size_t)k0 * es, w, true, true, false);
            update(F + ((size_t)k0 * ld + k0 + w) * es, ld, B + (size_t)k0 * es, B + (size_t)(k0 + w) * es, n - k0 - w, w);
        }
        // U: backward.
        int last = ((n - 1) / bs) * bs;
        for (int k0 = last; k0 >= 0; k0 -= bs) {
            int w = std::min(bs, n - k0);
            trsm(F + ((size_t)k0 * ld + k0) * es, B + (size_t)k0 * es, w, false, false, false);
            update(F + ((size_t)k0 * ld) * es, ld, B + (size_t)k0 * es, B, k0, w);
        }
    } else {
        // A^H = U^H L^H P^T: solve U^H (lower, non-unit), then L^H (upper,
        // unit), then undo the interchanges in reverse. The off-diagonal
        // blocks are the conjugate transposes of stored blocks, formed once.
        DMat fh(ctx, lu.cols, lu.rows, cplx, "the conjugate transpose of the factors");
        conj_transpose(ctx, fh, lu);
        const double* H = fh.p;
        const int ldh = fh.ld();
        for (int k0 = 0; k0 < n; k0 += bs) {
            int w = std::min(bs, n - k0);
            trsm(F + ((size_t)k0 * ld + k0) * es, B + (size_t)k0 * es, w, true, false, true);
            update(H + ((size_t)k0 * ldh + k0 + w) * es, ldh, B + (size_t)k0 * es, B + (size_t)(k0 + w) * es, n - k0 - w, w);
        }
        int last = ((n - 1) / bs) * bs;
        for (int k0 = last; k0 >= 0; k0 -= bs) {
            int w = std::min(bs, n - k0);
            trsm(F + ((size_t)k0 * ld + k0) * es, B + (size_t)k0 * es, w, false, true, true);
            update(H + ((size_t)k0 * ldh) * es, ldh, B + (size_t)k0 * es, B, k0, w);
        }
        launch_laswp(ctx, cplx, B, ldb, 0, nrhs, d_piv, 0, n, true);
    }
}

}  // namespace tns
