// Streaming kernels: elementwise updates, exact norms, the ell test's
// abs-power chain, and the narrow panel products behind normest1.
//
// All of these are HBM/L2-bound O(n^2) work. Where a result steers one of the
// reference's integer decisions (norms feeding d4/d6, the ell chain, the panel
// products inside normest1), the kernels keep the reference's summation order
// exactly -- one thread per output, accumulating in the reference's index
// order -- so that equal inputs give bit-equal decisions:
//   column sums      Norms.One            src/Tensile.Kernels/Norms.cs:11-26
//   row sums         Norms.Infinity       src/Tensile.Kernels/Norms.cs:50-66
//   complex moduli   Complex.Abs          src/Tensile/ComplexKernels.cs:111,144-180
//   abs-power chain  OneNormOfAbsolutePower src/Tensile/MatrixExponential.cs:468-505
//   A*X (axpy form)  PanelProduct.Apply    src/Tensile.Kernels/PanelProduct.cs:25-41
//   A^T*X (dot form) PanelProduct.ApplyTranspose :44-55 with ColumnOps.Dot's
//                    four 4-lane accumulators (src/Tensile.Kernels/ColumnOps.cs:35-65)

#include "device_util.cuh"
#include "tns_internal.h"

#include <algorithm>
#include <vector>

namespace tns {

namespace {

constexpr int kThreads = 256;

inline int blocks_for(long long n, int threads = kThreads) {
    long long b = (n + threads - 1) / threads;
    return (int)std::max(1LL, std::min(b, 148LL * 16));
}

__device__ __forceinline__ double mag(const double* a, size_t idx, bool cplx) {
    if (cplx) return cabs_net(a[2 * idx], a[2 * idx + 1]);
    return fabs(a[idx]);
}

// Scale: c := beta*c (beta == 0 overwrites), complex beta by the naive product.
__global__ void scale_kernel(double* c, int m, int n, int ldc, bool cplx, double br, double bi) {
    long long total = (long long)m * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        int i = (int)(e % m), j = (int)(e / m);
        size_t idx = (size_t)j * ldc + i;
        if (!cplx) {
            c[idx] = br == 0.0 ? 0.0 : mul_rn(c[idx], br);
        } else {
            double x = c[2 * idx], y = c[2 * idx + 1];
            if (br == 0.0 && bi == 0.0) {
                c[2 * idx] = 0.0;
                c[2 * idx + 1] = 0.0;
            } else {
                c[2 * idx] = sub_rn(mul_rn(br, x), mul_rn(bi, y));
                c[2 * idx + 1] = add_rn(mul_rn(bi, x), mul_rn(br, y));
            }
        }
    }
}

// dst := src * f over a flat range of doubles (each complex part on its own,
// ComplexKernels.Scale, src/Tensile/ComplexKernels.cs:132).
__global__ void scaled_copy_kernel(double* __restrict__ dst, const double* __restrict__ src, size_t count, double f) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x)
        dst[e] = mul_rn(src[e], f);
}

// t := t + s * f (AddScaled, src/Tensile/MatrixExponential.cs:546-558).
__global__ void add_scaled_kernel(double* __restrict__ t, const double* __restrict__ s, size_t count, double f) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x)
        t[e] = add_rn(t[e], mul_rn(s[e], f));
}

__global__ void identity_kernel(double* dst, int rows_p, int cols_p, int n, bool cplx, double f) {
    size_t total = (size_t)rows_p * cols_p * (cplx ? 2 : 1);
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        size_t el = cplx ? e / 2 : e;
        int i = (int)(el % rows_p), j = (int)(el / rows_p);
        bool re = !cplx || (e % 2 == 0);
        dst[e] = (i == j && i < n && re) ? f : 0.0;
    }
}

__global__ void pade_split_kernel(double* __restrict__ den, double* __restrict__ num, const double* __restrict__ v,
                                  const double* __restrict__ u, size_t count) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        den[e] = sub_rn(v[e], u[e]);
        num[e] = add_rn(v[e], u[e]);
    }
}

// One thread per column: sequential sum of moduli in row order.
__global__ void col_abs_sums_kernel(const double* __restrict__ a, int m, int n, int ld, bool cplx, double* __restrict__ out) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double* col = a + (size_t)j * ld * (cplx ? 2 : 1);
    double sum = 0.0;
    for (int i = 0; i < m; ++i) sum = add_rn(sum, mag(col, i, cplx));
    out[j] = sum;
}

// One thread per row: sequential sum over columns in column order.
__global__ void row_abs_sums_kernel(const double* __restrict__ a, int m, int n, int ld, bool cplx, double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    double sum = 0.0;
    for (int j = 0; j < n; ++j) sum = add_rn(sum, mag(a, (size_t)j * ld + i, cplx));
    out[i] = sum;
}

// Sum of squares per column (the reference's Frobenius accumulates one running
// total; this path is used only for diagnostics, not decisions).
__global__ void col_sq_sums_kernel(const double* __restrict__ a, int m, int n, int ld, bool cplx, double* __restrict__ out) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double* col = a + (size_t)j * ld * (cplx ? 2 : 1);
    double sum = 0.0;
    for (int i = 0; i < m * (cplx ? 2 : 1); ++i) sum = add_rn(sum, mul_rn(col[i], col[i]));
    out[j] = sum;
}

// Math.Max fold in index order (NaN propagates), single block.
__global__ void max_fold_kernel(const double* __restrict__ v, int n, double* __restrict__ out) {
    __shared__ double part[32];
    // Order-independent except for NaN and signed zero; v holds sums of
    // non-negative terms, so a tree with NaN propagation is exact.
    double best = 0.0;
    bool nan = false;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double x = v[i];
        if (isnan(x)) nan = true;
        else if (x > best) best = x;
    }
    for (int o = 16; o > 0; o >>= 1) {
        double other = __shfl_xor_sync(0xffffffffu, best, o);
        best = other > best ? other : best;
        nan = __any_sync(0xffffffffu, nan);
    }
    __shared__ int any_nan;
    if (threadIdx.x == 0) any_nan = 0;
    __syncthreads();
    if (nan && (threadIdx.x & 31) == 0) any_nan = 1;
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = part[w] > b ? part[w] : b;
        out[0] = any_nan ? __longlong_as_double(0x7ff8000000000000ll) : b;
    }
}

// |A| as a real n x n matrix (ld = n_p).
__global__ void moduli_kernel(const double* __restrict__ a, int n, int ld, bool cplx, double* __restrict__ mags) {
    size_t total = (size_t)ld * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % ld);
        mags[e] = i < n ? mag(a, e, cplx) : 0.0;
    }
}

// One pass of the chain: next[j] = sum_i row[i] * mags[i, j], sequential in i.
__global__ void abs_power_step_kernel(const double* __restrict__ mags, int n, int ld, const double* __restrict__ row,
                                      double* __restrict__ next) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double* col = mags + (size_t)j * ld;
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum = add_rn(sum, mul_rn(row[i], col[i]));
    next[j] = sum;
}

__global__ void fill_kernel(double* p, size_t count, double v) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x)
        p[e] = v;
}

// Y := A X in the axpy order of PanelProduct.Apply (PanelProduct.cs:25-41):
// y[i] accumulates x[j] * a[i, j] for j = 0..n-1 with two roundings per term,
// skipping x[j] == 0. The skip is kept exactly: a skipped term adds +0.0 to a
// sum that is never -0.0, which changes nothing, and it keeps 0 * inf out.
// Complex operator (LinearOperators.cs:262-282): four real sums per column,
// pr = Ar xr, pi = Ar xi, qr = Ai xr, qi = Ai xi, then (pr - qi, pi + qr).
// One thread per row covers all t <= TMAX columns, so A is read once per
// product; x is staged through shared memory.
template <int TMAX, bool CPLX>
__global__ void __launch_bounds__(128) panel_apply_kernel(const double* __restrict__ a, int n, int ld,
                                                          const double* __restrict__ x, int ldx,
                                                          double* __restrict__ y, int ldy, int t) {
    constexpr int CH = 64;  // rows of x staged per chunk
    constexpr int ES = CPLX ? 2 : 1;
    __shared__ double sx[CH * TMAX * ES];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool row_ok = i < n;
    double acc[TMAX][CPLX ? 4 : 1];
#pragma unroll
    for (int c = 0; c < TMAX; ++c)
#pragma unroll
        for (int q = 0; q < (CPLX ? 4 : 1); ++q) acc[c][q] = 0.0;
    for (int j0 = 0; j0 < n; j0 += CH) {
        const int len = min(CH, n - j0);
        __syncthreads();
        for (int e = threadIdx.x; e < len * t * ES; e += blockDim.x) {
            int c = e / (len * ES), r = e % (len * ES);
            sx[(c * CH) * ES + r] = x[((size_t)c * ldx + j0) * ES + r];
        }
        __syncthreads();
        if (!row_ok) continue;
        for (int jj = 0; jj < len; ++jj) {
            const size_t idx = (size_t)(j0 + jj) * ld + i;
            if (!CPLX) {
                const double aij = a[idx];
#pragma unroll
                for (int c = 0; c < TMAX; ++c) {
                    if (c < t) {
                        double s = sx[c * CH + jj];
                        double term = s != 0.0 ? mul_rn(s, aij) : 0.0;
                        acc[c][0] = add_rn(acc[c][0], term);
                    }
                }
            } else {
                const double2 aij = reinterpret_cast<const double2*>(a)[idx];
#pragma unroll
                for (int c = 0; c < TMAX; ++c) {
                    if (c < t) {
                        double sr = sx[(c * CH + jj) * 2], si = sx[(c * CH + jj) * 2 + 1];
                        bool nr = sr != 0.0, ni = si != 0.0;
                        acc[c][0] = add_rn(acc[c][0], nr ? mul_rn(sr, aij.x) : 0.0);  // pr
                        acc[c][2] = add_rn(acc[c][2], nr ? mul_rn(sr, aij.y) : 0.0);  // qr
                        acc[c][1] = add_rn(acc[c][1], ni ? mul_rn(si, aij.x) : 0.0);  // pi
                        acc[c][3] = add_rn(acc[c][3], ni ? mul_rn(si, aij.y) : 0.0);  // qi
                    }
                }
            }
        }
    }
    if (!row_ok) return;
#pragma unroll
    for (int c = 0; c < TMAX; ++c) {
        if (c >= t) continue;
        if (!CPLX) {
            y[(size_t)c * ldy + i] = acc[c][0];
        } else {
            reinterpret_cast<double2*>(y)[(size_t)c * ldy + i] =
                make_double2(sub_rn(acc[c][0], acc[c][3]), add_rn(acc[c][1], acc[c][2]));
        }
    }
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

// Y := A^T X (real) or A^H X (complex operator: pr = Ar^T xr, pi = Ar^T xi,
// qr = Ai^T xr, qi = Ai^T xi, then (pr + qi, pi - qr)), PanelProduct.ApplyTranspose
// (PanelProduct.cs:44-55): y[j] = Dot(a[:, j], x) in ColumnOps.Dot's order.
// One half-warp per output row j, covering all t <= TMAX columns, reading the
// interleaved complex data directly.
template <int TMAX, bool CPLX>
__global__ void panel_apply_t_kernel(const double* __restrict__ a, int n, int ld, const double* __restrict__ x,
                                     int ldx, double* __restrict__ y, int ldy, int t) {
    constexpr int NQ = CPLX ? 4 : 1;
    const long long half = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const int L = threadIdx.x & 15;
    const int base = threadIdx.x & 16;  // lane offset of this half in the warp
    // Inactive halves compute row 0 and drop it, so every shuffle sees a
    // converged warp.
    const bool active = half < n;
    const int j = active ? (int)half : 0;
    double acc[TMAX][NQ];
#pragma unroll
    for (int c = 0; c < TMAX; ++c)
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[c][q] = 0.0;
    const int W = 4;
    const int n16 = (n / (4 * W)) * (4 * W);
    const int n4 = n >= W ? n16 + ((n - n16) / W) * W : 0;
    auto add_term = [&](int i) {
        if (!CPLX) {
            double aij = a[(size_t)j * ld + i];
#pragma unroll
            for (int c = 0; c < TMAX; ++c)
                if (c < t) acc[c][0] = add_rn(acc[c][0], mul_rn(aij, x[(size_t)c * ldx + i]));
        } else {
            double2 aij = reinterpret_cast<const double2*>(a)[(size_t)j * ld + i];
#pragma unroll
            for (int c = 0; c < TMAX; ++c)
                if (c < t) {
                    double2 xc = reinterpret_cast<const double2*>(x)[(size_t)c * ldx + i];
                    acc[c][0] = add_rn(acc[c][0], mul_rn(aij.x, xc.x));  // pr
                    acc[c][1] = add_rn(acc[c][1], mul_rn(aij.x, xc.y));  // pi
                    acc[c][2] = add_rn(acc[c][2], mul_rn(aij.y, xc.x));  // qr
                    acc[c][3] = add_rn(acc[c][3], mul_rn(aij.y, xc.y));  // qi
                }
        }
    };
    double res[TMAX][NQ];
    if (n >= W) {
        for (int i = L; i < n16; i += 16) add_term(i);
        if (L < W)
            for (int i = n16 + L; i < n4; i += W) add_term(i);
#pragma unroll
        for (int c = 0; c < TMAX; ++c)
#pragma unroll
            for (int q = 0; q < NQ; ++q) res[c][q] = netdot_combine(acc[c][q], L, base);
    } else {
#pragma unroll
        for (int c = 0; c < TMAX; ++c)
#pragma unroll
            for (int q = 0; q < NQ; ++q) res[c][q] = 0.0;
    }
    if (!active || L != 0) return;
    // scalar tail, in order, by one lane
    for (int i = n4; i < n; ++i) {
        if (!CPLX) {
            double aij = a[(size_t)j * ld + i];
#pragma unroll
            for (int c = 0; c < TMAX; ++c)
                if (c < t) res[c][0] = add_rn(res[c][0], mul_rn(aij, x[(size_t)c * ldx + i]));
        } else {
            double2 aij = reinterpret_cast<const double2*>(a)[(size_t)j * ld + i];
#pragma unroll
            for (int c = 0; c < TMAX; ++c)
                if (c < t) {
                    double2 xc = reinterpret_cast<const double2*>(x)[(size_t)c * ldx + i];
                    res[c][0] = add_rn(res[c][0], mul_rn(aij.x, xc.x));
                    res[c][1] = add_rn(res[c][1], mul_rn(aij.x, xc.y));
                    res[c][2] = add_rn(res[c][2], mul_rn(aij.y, xc.x));
                    res[c][3] = add_rn(res[c][3], mul_rn(aij.y, xc.y));
                }
        }
    }
#pragma unroll
    for (int c = 0; c < TMAX; ++c) {
        if (c >= t) continue;
        if (!CPLX)
            y[(size_t)c * ldy + j] = res[c][0];
        else
            reinterpret_cast<double2*>(y)[(size_t)c * ldy + j] =
                make_double2(add_rn(res[c][0], res[c][3]), sub_rn(res[c][1], res[c][2]));
    }
}

__global__ void shift_diag_kernel(double* a, int n, int ld, bool cplx, double dre, double dim) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!cplx) {
        a[(size_t)i * ld + i] = add_rn(a[(size_t)i * ld + i], dre);
    } else {
        double2* p = reinterpret_cast<double2*>(a) + (size_t)i * ld + i;
        double2 z = *p;
        *p = make_double2(add_rn(z.x, dre), add_rn(z.y, dim));
    }
}

// Trace: sequential sum (one thread), as the reference's loop.
__global__ void trace_kernel(const double* a, int n, int ld, bool cplx, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double re = 0.0, im = 0.0;
    for (int i = 0; i < n; ++i) {
        if (!cplx) {
            re = add_rn(re, a[(size_t)i * ld + i]);
        } else {
            double2 z = reinterpret_cast<const double2*>(a)[(size_t)i * ld + i];
            re = add_rn(re, z.x);
            im = add_rn(im, z.y);
        }
    }
    out[0] = re;
    out[1] = im;
}

double fetch_scalar(Context& ctx, const double* d) {
    double h = 0.0;
    TNS_CUDA(cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    return h;
}

}  // namespace

// ---------------------------------------------------------------------------

void scale_inplace(Context& ctx, void* c, int m, int n, int ldc, bool cplx, double br, double bi) {
    if (br == 1.0 && bi == 0.0) return;
    if ((long long)m * n == 0) return;
    scale_kernel<<<blocks_for((long long)m * n), kThreads, 0, ctx.stream>>>(static_cast<double*>(c), m, n, ldc, cplx, br, bi);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void scaled_copy(Context& ctx, DMat& dst, const DMat& src, double f) {
    size_t count = src.bytes() / 8;
    scaled_copy_kernel<<<blocks_for((long long)count), kThreads, 0, ctx.stream>>>(dst.p, src.p, count, f);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void add_scaled(Context& ctx, DMat& t, const DMat& s, double f) {
    size_t count = s.bytes() / 8;
    add_scaled_kernel<<<blocks_for((long long)count), kThreads, 0, ctx.stream>>>(t.p, s.p, count, f);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void set_identity(Context& ctx, DMat& dst, double f) {
    size_t total = dst.bytes() / 8;
    identity_kernel<<<blocks_for((long long)total), kThreads, 0, ctx.stream>>>(dst.p, dst.rows_p, dst.cols_p, dst.rows,
                                                                               dst.cplx, f);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void pade_split(Context& ctx, DMat& den, DMat& num, const DMat& v, const DMat& u) {
    size_t count = v.bytes() / 8;
    pade_split_kernel<<<blocks_for((long long)count), kThreads, 0, ctx.stream>>>(den.p, num.p, v.p, u.p, count);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

double norm1(Context& ctx, const DMat& a) {
    if (a.rows == 0 || a.cols == 0) return 0.0;
    DBuf sums(ctx, sizeof(double) * (a.cols + 1));
    col_abs_sums_kernel<<<(a.cols + 127) / 128, 128, 0, ctx.stream>>>(a.p, a.rows, a.cols, a.ld(), a.cplx, sums.as<double>());
    max_fold_kernel<<<1, 256, 0, ctx.stream>>>(sums.as<double>(), a.cols, sums.as<double>() + a.cols);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches += 2;
    return fetch_scalar(ctx, sums.as<double>() + a.cols);
}

double norminf(Context& ctx, const DMat& a) {
    if (a.rows == 0 || a.cols == 0) return 0.0;
    DBuf sums(ctx, sizeof(double) * (a.rows + 1));
    row_abs_sums_kernel<<<(a.rows + 127) / 128, 128, 0, ctx.stream>>>(a.p, a.rows, a.cols, a.ld(), a.cplx, sums.as<double>());
    max_fold_kernel<<<1, 256, 0, ctx.stream>>>(sums.as<double>(), a.rows, sums.as<double>() + a.rows);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches += 2;
    return fetch_scalar(ctx, sums.as<double>() + a.rows);
}

double normfro(Context& ctx, const DMat& a) {
    if (a.rows == 0 || a.cols == 0) return 0.0;
    DBuf sums(ctx, sizeof(double) * a.cols);
    col_sq_sums_kernel<<<(a.cols + 127) / 128, 128, 0, ctx.stream>>>(a.p, a.rows, a.cols, a.ld(), a.cplx, sums.as<double>());
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
    std::vector<double> h(a.cols);
    TNS_CUDA(cudaMemcpyAsync(h.data(), sums.p, sizeof(double) * a.cols, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    double total = 0.0;
    for (double v : h) total += v;
    return std::sqrt(total);
}

double one_norm_abs_power(Context& ctx, const DMat& a, int p) {
    int n = a.rows;
    int ld = a.ld();
    DBuf mags(ctx, sizeof(double) * (size_t)ld * n);
    DBuf vecs(ctx, sizeof(double) * (2 * (size_t)n + 1));
    double* row = vecs.as<double>();
    double* next = row + n;
    moduli_kernel<<<blocks_for((long long)ld * n), kThreads, 0, ctx.stream>>>(a.p, n, ld, a.cplx, mags.as<double>());
    fill_kernel<<<blocks_for(n), kThreads, 0, ctx.stream>>>(row, n, 1.0);
    ctx.kernel_launches += 2;
    for (int step = 0; step < p; ++step) {
        abs_power_step_kernel<<<(n + 127) / 128, 128, 0, ctx.stream>>>(mags.as<double>(), n, ld, row, next);
        std::swap(row, next);
        ctx.kernel_launches++;
    }
    max_fold_kernel<<<1, 256, 0, ctx.stream>>>(row, n, vecs.as<double>() + 2 * (size_t)n);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
    return fetch_scalar(ctx, vecs.as<double>() + 2 * (size_t)n);
}

namespace {
template <int TMAX, bool CPLX>
void launch_panel(Context& ctx, const DMat& a, const double* x, int ldx, double* y, int ldy, int t, bool adjoint) {
    int n = a.rows;
    if (!adjoint) {
        panel_apply_kernel<TMAX, CPLX><<<(n + 127) / 128, 128, 0, ctx.stream>>>(a.p, n, a.ld(), x, ldx, y, ldy, t);
    } else {
        long long threads = (long long)n * 16;
        panel_apply_t_kernel<TMAX, CPLX><<<(int)((threads + 255) / 256), 256, 0, ctx.stream>>>(a.p, n, a.ld(), x, ldx, y,
                                                                                               ldy, t);
    }
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}
template <bool CPLX>
void panel_dispatch(Context& ctx, const DMat& a, const double* x, int ldx, double* y, int ldy, int t, bool adjoint) {
    if (t <= 2) launch_panel<2, CPLX>(ctx, a, x, ldx, y, ldy, t, adjoint);
    else if (t <= 4) launch_panel<4, CPLX>(ctx, a, x, ldx, y, ldy, t, adjoint);
    else if (t <= 8) launch_panel<8, CPLX>(ctx, a, x, ldx, y, ldy, t, adjoint);
    else launch_panel<16, CPLX>(ctx, a, x, ldx, y, ldy, t, adjoint);
}
}  // namespace

void panel_product(Context& ctx, const DMat& a, const double* x, int ldx, double* y, int ldy, int t, bool adjoint) {
    if (a.rows == 0 || t == 0) return;
    // Wider panels run as successive blocks of 16 columns; each column's
    // arithmetic is independent of the others.
    for (int c0 = 0; c0 < t; c0 += 16) {
        int tc = std::min(16, t - c0);
        size_t es = a.cplx ? 2 : 1;
        const double* xc = x + (size_t)c0 * ldx * es;
        double* yc = y + (size_t)c0 * ldy * es;
        if (a.cplx) panel_dispatch<true>(ctx, a, xc, ldx, yc, ldy, tc, adjoint);
        else panel_dispatch<false>(ctx, a, xc, ldx, yc, ldy, tc, adjoint);
    }
}

void shift_diagonal(Context& ctx, DMat& a, double dre, double dim) {
    if (a.rows == 0) return;
    shift_diag_kernel<<<(a.rows + 127) / 128, 128, 0, ctx.stream>>>(a.p, a.rows, a.ld(), a.cplx, dre, dim);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void trace(Context& ctx, const DMat& a, double* re, double* im) {
    DBuf out(ctx, 2 * sizeof(double));
    trace_kernel<<<1, 32, 0, ctx.stream>>>(a.p, a.rows, a.ld(), a.cplx, out.as<double>());
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
    double h[2];
    TNS_CUDA(cudaMemcpyAsync(h, out.p, sizeof(h), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    *re = h[0];
    *im = h[1];
}

}  // namespace tns
