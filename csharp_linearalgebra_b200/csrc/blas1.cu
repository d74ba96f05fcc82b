// Streaming kernels: elementwise updates, exact norms, the ell test's
// abs-power chain, and the narrow panel products behind normest1. Every
// kernel takes a Batch<D>: one launch serves one matrix or a whole batch.
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

#include "batch.cuh"
#include "device_util.cuh"
#include "tns_internal.h"

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

namespace tns {

namespace {

constexpr int kThreads = 256;

inline int blocks_for(long long n, int threads = kThreads, int cap = 148 * 16) {
    long long b = (n + threads - 1) / threads;
    return (int)std::max(1LL, std::min(b, (long long)cap));
}

__device__ __forceinline__ double mag(const double* a, size_t idx, bool cplx) {
    if (cplx) return cabs_net(a[2 * idx], a[2 * idx + 1]);
    return fabs(a[idx]);
}

// ---- elementwise ------------------------------------------------------------

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

// Elementwise operations over a matrix's whole padded extent (zeros in the
// padding stay zero):
//   kScaledCopy  dst = s1 * f          (Scaled, MatrixExponential.cs:528-543;
//                                       complex parts scaled on their own)
//   kAddScaled   dst = dst + s1 * f    (AddScaled, :546-558)
//   kIdentity    dst = f I on the valid diagonal (Identity, :518-525)
//   kPadeSplit   dst = s1 - s2, dst2 = s1 + s2 (SolvePade, :381-393)
enum EwOp : int { kScaledCopy = 0, kAddScaled = 1, kIdentity = 2, kPadeSplit = 3 };

__global__ void ew_kernel(const __grid_constant__ Batch<EwDesc> b) {
    const EwDesc& d = batch_item(b, blockIdx.y);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < d.count; e += stride) {
        switch (d.op) {
            case kScaledCopy: d.dst[e] = mul_rn(d.s1[e], d.f); break;
            case kAddScaled: d.dst[e] = add_rn(d.dst[e], mul_rn(d.s1[e], d.f)); break;
            case kIdentity: {
                size_t el = d.cplx ? e / 2 : e;
                int i = (int)(el % d.rows_p), j = (int)(el / d.rows_p);
                bool re = !d.cplx || (e % 2 == 0);
                d.dst[e] = (i == j && i < d.n && re) ? d.f : 0.0;
                break;
            }
            case kPadeSplit:
                d.dst[e] = sub_rn(d.s1[e], d.s2[e]);
                d.dst2[e] = add_rn(d.s1[e], d.s2[e]);
                break;
        }
    }
}

// The Pade numerator's parts in one pass over the elements
// (EvaluateDegree13 / EvaluateLowDegree, MatrixExponential.cs:284-360): each
// element goes through exactly the Scaled / AddScaled / Identity steps of the
// reference, in its order, so every rounding is the same; the scaled powers
// B^2, B^4 are never stored.
//   degree 13: B = f A, B6 = f^6 A^6 (kept for the products), and
//     inner      = c13 B6 + c11 B4 + c9 B2
//     w          = c1 I + c3 B2 + c5 B4 + c7 B6
//     inner_even = c12 B6 + c10 B4 + c8 B2
//     v          = c0 I + c2 B2 + c4 B4 + c6 B6
//   degree 3..9: w = c1 I + c3 A2 (+ c5 A4 + c7 A6 + c9 A8), v likewise.
__global__ void pade_assemble_kernel(const __grid_constant__ Batch<PadeDesc> bt) {
    const PadeDesc& d = batch_item(bt, blockIdx.y);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const double* c = d.c;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < d.count; e += stride) {
        const size_t el = d.cplx ? e / 2 : e;
        const int i = (int)(el % d.rows_p), j = (int)(el / d.rows_p);
        const bool diag = i == j && i < d.n && (!d.cplx || (e % 2 == 0));
        if (d.degree == 13) {
            const double x2 = mul_rn(d.a2[e], d.f2), x4 = mul_rn(d.a4[e], d.f4), x6 = mul_rn(d.a6[e], d.f6);
            d.b[e] = mul_rn(d.a[e], d.f);
            d.b6[e] = x6;
            d.inner[e] = add_rn(add_rn(mul_rn(x6, c[13]), mul_rn(x4, c[11])), mul_rn(x2, c[9]));
            d.w[e] = add_rn(add_rn(add_rn(diag ? c[1] : 0.0, mul_rn(x2, c[3])), mul_rn(x4, c[5])), mul_rn(x6, c[7]));
            d.inner_even[e] = add_rn(add_rn(mul_rn(x6, c[12]), mul_rn(x4, c[10])), mul_rn(x2, c[8]));
            d.v[e] = add_rn(add_rn(add_rn(diag ? c[0] : 0.0, mul_rn(x2, c[2])), mul_rn(x4, c[4])), mul_rn(x6, c[6]));
        } else {
            double w = add_rn(diag ? c[1] : 0.0, mul_rn(d.a2[e], c[3]));
            double v = add_rn(diag ? c[0] : 0.0, mul_rn(d.a2[e], c[2]));
            if (d.degree >= 5) {
                w = add_rn(w, mul_rn(d.a4[e], c[5]));
                v = add_rn(v, mul_rn(d.a4[e], c[4]));
            }
            if (d.degree >= 7) {
                w = add_rn(w, mul_rn(d.a6[e], c[7]));
                v = add_rn(v, mul_rn(d.a6[e], c[6]));
            }
            if (d.degree == 9) {
                w = add_rn(w, mul_rn(d.a8[e], c[9]));
                v = add_rn(v, mul_rn(d.a8[e], c[8]));
            }
            d.w[e] = w;
            d.v[e] = v;
        }
    }
}

// ---- norms ------------------------------------------------------------------

// One warp per column: lanes load 32 consecutive entries (coalesced) and
// form their moduli in parallel; the sum then takes them one by one in row
// order (each broadcast by a shuffle), the same sequential sum as one thread
// walking the column.
template <bool CPLX>
__global__ void col_abs_sums_kernel(const __grid_constant__ Batch<SumDesc> b) {
    const SumDesc& d = batch_item(b, blockIdx.y);
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (j >= d.n) return;  // the whole warp
    const double* col = d.a + (size_t)j * d.ld * (CPLX ? 2 : 1);
    double sum = 0.0;
    for (int i0 = 0; i0 < d.m; i0 += 32) {
        const double v = i0 + lane < d.m ? mag(col, i0 + lane, CPLX) : 0.0;
        const int cnt = min(32, d.m - i0);
        for (int l = 0; l < cnt; ++l) sum = add_rn(sum, __shfl_sync(0xffffffffu, v, l));
    }
    if (lane == 0) d.out[j] = sum;
}

// One thread per row: sequential sum over columns in column order.
template <bool CPLX>
__global__ void row_abs_sums_kernel(const __grid_constant__ Batch<SumDesc> b) {
    const SumDesc& d = batch_item(b, blockIdx.y);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.m) return;
    double sum = 0.0;
    for (int j = 0; j < d.n; ++j) sum = add_rn(sum, mag(d.a, (size_t)j * d.ld + i, CPLX));
    d.out[i] = sum;
}

// Sum of squares per column (diagnostic Frobenius only; no decision uses it).
__global__ void col_sq_sums_kernel(const double* __restrict__ a, int m, int n, int ld, bool cplx, double* __restrict__ out) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double* col = a + (size_t)j * ld * (cplx ? 2 : 1);
    double sum = 0.0;
    for (int i = 0; i < m * (cplx ? 2 : 1); ++i) sum = add_rn(sum, mul_rn(col[i], col[i]));
    out[j] = sum;
}

// Math.Max fold of non-negative sums (NaN propagates): a tree reduction gives
// the sequential fold's result, since max is order-independent here. One
// block per item.
__global__ void max_fold_kernel(const __grid_constant__ Batch<SumDesc> b) {
    const SumDesc& d = batch_item(b, blockIdx.x);
    __shared__ double part[32];
    __shared__ int any_nan;
    if (threadIdx.x == 0) any_nan = 0;
    __syncthreads();
    double best = 0.0;
    bool nan = false;
    for (int i = threadIdx.x; i < d.n; i += blockDim.x) {
        double x = d.a[i];
        if (isnan(x)) nan = true;
        else if (x > best) best = x;
    }
    for (int o = 16; o > 0; o >>= 1) {
        double other = __shfl_xor_sync(0xffffffffu, best, o);
        best = other > best ? other : best;
    }
    if (nan) atomicOr(&any_nan, 1);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = part[w] > r ? part[w] : r;
        d.out[0] = any_nan ? __longlong_as_double(0x7ff8000000000000ll) : r;
    }
}

// ---- the ell test's chain -----------------------------------------------------

// |A| as a real matrix (ld = n_p); row := ones.
template <bool CPLX>
__global__ void moduli_kernel(const __grid_constant__ Batch<ChainDesc> b) {
    const ChainDesc& d = batch_item(b, blockIdx.y);
    size_t total = (size_t)d.ld * d.n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e % d.ld);
        d.mags[e] = i < d.n ? mag(d.a, e, CPLX) : 0.0;
        if (e < (size_t)d.n) d.row[e] = 1.0;
    }
}

// One pass: next[j] = sum_i row[i] * mags[i, j], sequential in i. One warp
// per 32 columns: each 32-row chunk of them is read by 32 coalesced loads
// (one column each, a row per lane, the next chunk's loads issued before this
// chunk is used), transposed through shared memory, and lane c continues
// column c's sum over the chunk's rows in order: one thread's sequential sum
// per column, as before, with the reads in whole sectors.
constexpr int kChainWarps = 4;
__global__ void __launch_bounds__(32 * kChainWarps) abs_power_step_kernel(const __grid_constant__ Batch<ChainDesc> b,
                                                                          int parity) {
    const ChainDesc& d = batch_item(b, blockIdx.y);
    __shared__ double tile[kChainWarps][32][33];
    __shared__ double rowv[kChainWarps][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j0 = (blockIdx.x * kChainWarps + warp) * 32;
    if (j0 >= d.n) return;  // the whole warp; only warp-level synchronisation below
    const double* row = parity ? d.next : d.row;
    double* out = parity ? d.row : d.next;
    const int ncol = min(32, d.n - j0);
    double cur[32], nxt[32];
    auto load = [&](int i0, double (&v)[32]) {
        const int i = i0 + lane;
#pragma unroll
        for (int c = 0; c < 32; ++c) v[c] = (c < ncol && i < d.n) ? d.mags[(size_t)(j0 + c) * d.ld + i] : 0.0;
    };
    double sum = 0.0;
    load(0, cur);
    for (int i0 = 0; i0 < d.n; i0 += 32) {
        if (i0 + 32 < d.n) load(i0 + 32, nxt);
#pragma unroll
        for (int c = 0; c < 32; ++c) tile[warp][c][lane] = cur[c];
        rowv[warp][lane] = i0 + lane < d.n ? row[i0 + lane] : 0.0;
        __syncwarp();
        const int cnt = min(32, d.n - i0);
        if (lane < ncol)
            for (int r = 0; r < cnt; ++r) sum = add_rn(sum, mul_rn(rowv[warp][r], tile[warp][lane][r]));
        __syncwarp();
#pragma unroll
        for (int c = 0; c < 32; ++c) cur[c] = nxt[c];
    }
    if (lane < ncol) out[j0 + lane] = sum;
}

// ---- normest1 panel products ------------------------------------------------

// Y := A X in the axpy order of PanelProduct.Apply (PanelProduct.cs:25-41):
// y[i] accumulates x[j] * a[i, j] for j = 0..n-1 with two roundings per term,
// skipping x[j] == 0. The skip is kept exactly: a skipped term adds +0.0 to a
// sum that is never -0.0, which changes nothing, and it keeps 0 * inf out.
// Complex operator (LinearOperators.cs:262-282): four real sums per column,
// pr = Ar xr, pi = Ar xi, qr = Ai xr, qi = Ai xi, then (pr - qi, pi + qr).
// TPR threads share a row, thread `sub` covering columns sub, sub + TPR, ...
// (each (row, column) sum stays one thread's chain); the row's A entries are
// one load for all of them, so A is read once per product. x is staged
// through shared memory.
template <int TMAX, bool CPLX, int TPR>
__global__ void __launch_bounds__(128) panel_apply_kernel(const __grid_constant__ Batch<PanelDesc> b) {
    constexpr int RPB = 128 / TPR;       // rows per block
    constexpr int CPT = TMAX / TPR;      // columns per thread
    const PanelDesc& d = batch_item(b, blockIdx.y);
    const int n = d.n, t = d.t;
    if ((int)(blockIdx.x * RPB) >= n) return;  // whole block past this item
    constexpr int CH = 64;                     // rows of x staged per chunk
    constexpr int ES = CPLX ? 2 : 1;
    __shared__ double sx[CH * TMAX * ES];
    const int i = blockIdx.x * RPB + threadIdx.x / TPR;
    const int sub = threadIdx.x % TPR;
    const bool row_ok = i < n;
    double acc[CPT][CPLX ? 4 : 1];
#pragma unroll
    for (int q = 0; q < CPT; ++q)
#pragma unroll
        for (int z = 0; z < (CPLX ? 4 : 1); ++z) acc[q][z] = 0.0;
    for (int j0 = 0; j0 < n; j0 += CH) {
        const int len = min(CH, n - j0);
        __syncthreads();
        for (int e = threadIdx.x; e < len * t * ES; e += blockDim.x) {
            int c = e / (len * ES), r = e % (len * ES);
            sx[(c * CH) * ES + r] = d.x[((size_t)c * d.ldx + j0) * ES + r];
        }
        __syncthreads();
        if (!row_ok) continue;
        // The sums stay sequential in j; the loads of A run U columns ahead
        // of them, so each thread keeps U loads in flight.
        constexpr int U = 16;
        using AE = typename std::conditional<CPLX, double2, double>::type;
        const AE* arow = reinterpret_cast<const AE*>(d.a) + (size_t)j0 * d.ld + i;
        for (int jb = 0; jb < len; jb += U) {
            AE av[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (jb + u < len) av[u] = arow[(size_t)(jb + u) * d.ld];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (jb + u >= len) break;
                const int jj = jb + u;
#pragma unroll
                for (int q = 0; q < CPT; ++q) {
                    const int c = sub + q * TPR;
                    if (c >= t) continue;
                    if constexpr (!CPLX) {
                        double sv = sx[c * CH + jj];
                        double term = sv != 0.0 ? mul_rn(sv, av[u]) : 0.0;
                        acc[q][0] = add_rn(acc[q][0], term);
                    } else {
                        const double2 aij = av[u];
                        double sr = sx[(c * CH + jj) * 2], si = sx[(c * CH + jj) * 2 + 1];
                        bool nr = sr != 0.0, ni = si != 0.0;
                        acc[q][0] = add_rn(acc[q][0], nr ? mul_rn(sr, aij.x) : 0.0);  // pr
                        acc[q][2] = add_rn(acc[q][2], nr ? mul_rn(sr, aij.y) : 0.0);  // qr
                        acc[q][1] = add_rn(acc[q][1], ni ? mul_rn(si, aij.x) : 0.0);  // pi
                        acc[q][3] = add_rn(acc[q][3], ni ? mul_rn(si, aij.y) : 0.0);  // qi
                    }
                }
            }
        }
    }
    if (!row_ok) return;
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
        const int c = sub + q * TPR;
        if (c >= t) continue;
        if (!CPLX) {
            d.y[(size_t)c * d.ldy + i] = acc[q][0];
        } else {
            reinterpret_cast<double2*>(d.y)[(size_t)c * d.ldy + i] =
                make_double2(sub_rn(acc[q][0], acc[q][3]), add_rn(acc[q][1], acc[q][2]));
        }
    }
}

// Y := A^T X (real) or A^H X (complex operator: pr = Ar^T xr, pi = Ar^T xi,
// qr = Ai^T xr, qi = Ai^T xi, then (pr + qi, pi - qr)), PanelProduct.ApplyTranspose
// (PanelProduct.cs:44-55): y[j] = Dot(a[:, j], x) in ColumnOps.Dot's order.
// One half-warp per output row j, covering all t <= TMAX columns, reading the
// interleaved complex data directly.
template <int TMAX, bool CPLX>
__global__ void panel_apply_t_kernel(const __grid_constant__ Batch<PanelDesc> b) {
    const PanelDesc& d = batch_item(b, blockIdx.y);
    const int n = d.n, t = d.t;
    if ((long long)blockIdx.x * blockDim.x >= (long long)n * 16) return;  // whole block past this item
    constexpr int NQ = CPLX ? 4 : 1;
    const long long half = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const int L = threadIdx.x & 15;
    const int base = threadIdx.x & 16;  // lane offset of this half in the warp
    // Inactive halves compute row 0 and drop it, so every shuffle sees a
    // converged warp.
    const bool active = half < n;
    const int j = active ? (int)half : 0;
    const double* a = d.a;
    const double* x = d.x;
    const int ld = d.ld, ldx = d.ldx;
    double acc[TMAX][NQ];
#pragma unroll
    for (int c = 0; c < TMAX; ++c)
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[c][q] = 0.0;
    const int W = 4;
    const int n16 = (n / (4 * W)) * (4 * W);
    const int n4 = n >= W ? n16 + ((n - n16) / W) * W : 0;
    auto add_term = [&](double (&r)[TMAX][NQ], int i) {
        if (!CPLX) {
            double aij = a[(size_t)j * ld + i];
#pragma unroll
            for (int c = 0; c < TMAX; ++c)
                if (c < t) r[c][0] = add_rn(r[c][0], mul_rn(aij, x[(size_t)c * ldx + i]));
        } else {
            double2 aij = reinterpret_cast<const double2*>(a)[(size_t)j * ld + i];
#pragma unroll
            for (int c = 0; c < TMAX; ++c)
                if (c < t) {
                    double2 xc = reinterpret_cast<const double2*>(x)[(size_t)c * ldx + i];
                    r[c][0] = add_rn(r[c][0], mul_rn(aij.x, xc.x));  // pr
                    r[c][1] = add_rn(r[c][1], mul_rn(aij.x, xc.y));  // pi
                    r[c][2] = add_rn(r[c][2], mul_rn(aij.y, xc.x));  // qr
                    r[c][3] = add_rn(r[c][3], mul_rn(aij.y, xc.y));  // qi
                }
        }
    };
    double res[TMAX][NQ];
    if (n >= W) {
        for (int i = L; i < n16; i += 16) add_term(acc, i);
        if (L < W)
            for (int i = n16 + L; i < n4; i += W) add_term(acc, i);
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
    for (int i = n4; i < n; ++i) add_term(res, i);  // scalar tail, in order
#pragma unroll
    for (int c = 0; c < TMAX; ++c) {
        if (c >= t) continue;
        if (!CPLX)
            d.y[(size_t)c * d.ldy + j] = res[c][0];
        else
            reinterpret_cast<double2*>(d.y)[(size_t)c * d.ldy + j] =
                make_double2(add_rn(res[c][0], res[c][3]), sub_rn(res[c][1], res[c][2]));
    }
}

// ---- small single-matrix helpers ----------------------------------------------

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

template <int TMAX, bool CPLX>
void launch_panel(Context& ctx, std::vector<PanelDesc>& v, bool adjoint) {
    int nmax = 0;
    for (auto& d : v) nmax = std::max(nmax, d.n);
    if (nmax == 0) return;
    Batch<PanelDesc> b = make_batch(ctx, v);
    if (!adjoint) {
        // Narrow panels (the estimator's two or four columns): one thread per
        // (row, column), twice or four times the threads of one per row.
        constexpr int TPR = TMAX <= 4 ? TMAX : 1;
        dim3 grid((nmax + 128 / TPR - 1) / (128 / TPR), b.count);
        panel_apply_kernel<TMAX, CPLX, TPR><<<grid, 128, 0, ctx.stream>>>(b);
    } else {
        long long threads = (long long)nmax * 16;
        dim3 grid((unsigned)((threads + 255) / 256), b.count);
        panel_apply_t_kernel<TMAX, CPLX><<<grid, 256, 0, ctx.stream>>>(b);
    }
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

}  // namespace

// ---------------------------------------------------------------------------
// Batched host entry points
// ---------------------------------------------------------------------------

void pade_assemble_batch(Context& ctx, std::vector<PadeDesc>& v) {
    if (v.empty()) return;
    long long maxc = 0;
    for (auto& d : v) maxc = std::max(maxc, (long long)d.count);
    if (maxc == 0) return;
    Batch<PadeDesc> b = make_batch(ctx, v);
    int bx = blocks_for(maxc, kThreads, std::max(1, 148 * 8 / (int)v.size()) + 1);
    pade_assemble_kernel<<<dim3(bx, b.count), kThreads, 0, ctx.stream>>>(b);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void ew_batch(Context& ctx, std::vector<EwDesc>& v) {
    if (v.empty()) return;
    long long maxc = 0;
    for (auto& d : v) maxc = std::max(maxc, (long long)d.count);
    if (maxc == 0) return;
    Batch<EwDesc> b = make_batch(ctx, v);
    int bx = blocks_for(maxc, kThreads, std::max(1, 148 * 8 / (int)v.size()) + 1);
    ew_kernel<<<dim3(bx, b.count), kThreads, 0, ctx.stream>>>(b);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

EwDesc ew_scaled_copy(DMat& dst, const DMat& src, double f) {
    EwDesc d{};
    d.op = kScaledCopy;
    d.dst = dst.p;
    d.s1 = src.p;
    d.count = src.bytes() / 8;
    d.f = f;
    return d;
}
EwDesc ew_add_scaled(DMat& t, const DMat& s, double f) {
    EwDesc d{};
    d.op = kAddScaled;
    d.dst = t.p;
    d.s1 = s.p;
    d.count = s.bytes() / 8;
    d.f = f;
    return d;
}
EwDesc ew_identity(DMat& dst, double f) {
    EwDesc d{};
    d.op = kIdentity;
    d.dst = dst.p;
    d.count = dst.bytes() / 8;
    d.f = f;
    d.rows_p = dst.rows_p;
    d.n = dst.rows;
    d.cplx = dst.cplx ? 1 : 0;
    return d;
}
EwDesc ew_pade_split(DMat& den, DMat& num, const DMat& v, const DMat& u) {
    EwDesc d{};
    d.op = kPadeSplit;
    d.dst = den.p;
    d.dst2 = num.p;
    d.s1 = v.p;
    d.s2 = u.p;
    d.count = v.bytes() / 8;
    return d;
}

std::vector<double> norm1_batch(Context& ctx, const std::vector<const DMat*>& mats) {
    std::vector<double> out(mats.size(), 0.0);
    if (mats.empty()) return out;
    bool cplx = mats[0]->cplx;
    size_t total = 0;
    for (auto* m : mats) total += (size_t)m->cols + 1;
    DBuf buf(ctx, sizeof(double) * std::max<size_t>(total, 1));
    std::vector<SumDesc> sums, folds;
    size_t off = 0;
    int nmax = 0;
    for (auto* m : mats) {
        double* base = buf.as<double>() + off;
        sums.push_back(SumDesc{m->p, m->rows, m->cols, m->ld(), base});
        folds.push_back(SumDesc{base, 0, m->cols, 0, base + m->cols});
        off += (size_t)m->cols + 1;
        nmax = std::max(nmax, m->cols);
    }
    Batch<SumDesc> bs = make_batch(ctx, sums);
    dim3 grid((nmax + 3) / 4, bs.count);  // 4 warps, one column each
    if (cplx) col_abs_sums_kernel<true><<<grid, 128, 0, ctx.stream>>>(bs);
    else col_abs_sums_kernel<false><<<grid, 128, 0, ctx.stream>>>(bs);
    Batch<SumDesc> bf = make_batch(ctx, folds);
    max_fold_kernel<<<bf.count, 256, 0, ctx.stream>>>(bf);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches += 2;
    std::vector<double> host(total);
    TNS_CUDA(cudaMemcpyAsync(host.data(), buf.p, sizeof(double) * total, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    off = 0;
    for (size_t k = 0; k < mats.size(); ++k) {
        out[k] = (mats[k]->rows == 0 || mats[k]->cols == 0) ? 0.0 : host[off + mats[k]->cols];
        off += (size_t)mats[k]->cols + 1;
    }
    return out;
}

std::vector<double> norminf_batch(Context& ctx, const std::vector<const DMat*>& mats) {
    std::vector<double> out(mats.size(), 0.0);
    if (mats.empty()) return out;
    bool cplx = mats[0]->cplx;
    size_t total = 0;
    for (auto* m : mats) total += (size_t)m->rows + 1;
    DBuf buf(ctx, sizeof(double) * std::max<size_t>(total, 1));
    std::vector<SumDesc> sums, folds;
    size_t off = 0;
    int mmax = 0;
    for (auto* m : mats) {
        double* base = buf.as<double>() + off;
        sums.push_back(SumDesc{m->p, m->rows, m->cols, m->ld(), base});
        folds.push_back(SumDesc{base, 0, m->rows, 0, base + m->rows});
        off += (size_t)m->rows + 1;
        mmax = std::max(mmax, m->rows);
    }
    Batch<SumDesc> bs = make_batch(ctx, sums);
    dim3 grid((mmax + 127) / 128, bs.count);
    if (cplx) row_abs_sums_kernel<true><<<grid, 128, 0, ctx.stream>>>(bs);
    else row_abs_sums_kernel<false><<<grid, 128, 0, ctx.stream>>>(bs);
    Batch<SumDesc> bf = make_batch(ctx, folds);
    max_fold_kernel<<<bf.count, 256, 0, ctx.stream>>>(bf);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches += 2;
    std::vector<double> host(total);
    TNS_CUDA(cudaMemcpyAsync(host.data(), buf.p, sizeof(double) * total, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    off = 0;
    for (size_t k = 0; k < mats.size(); ++k) {
        out[k] = (mats[k]->rows == 0 || mats[k]->cols == 0) ? 0.0 : host[off + mats[k]->rows];
        off += (size_t)mats[k]->rows + 1;
    }
    return out;
}

std::vector<double> abs_power_batch(Context& ctx, const std::vector<const DMat*>& mats, int p) {
    std::vector<double> out(mats.size(), 0.0);
    if (mats.empty()) return out;
    bool cplx = mats[0]->cplx;
    size_t mag_total = 0, vec_total = 0;
    for (auto* m : mats) {
        mag_total += (size_t)m->ld() * m->rows;
        vec_total += 2 * (size_t)m->rows + 1;
    }
    DBuf mags(ctx, sizeof(double) * std::max<size_t>(mag_total, 1));
    DBuf vecs(ctx, sizeof(double) * vec_total);
    std::vector<ChainDesc> chains;
    std::vector<SumDesc> folds;
    size_t mo = 0, vo = 0;
    int nmax = 0;
    long long emax = 0;
    for (auto* m : mats) {
        double* row = vecs.as<double>() + vo;
        ChainDesc c{m->p, m->rows, m->ld(), mags.as<double>() + mo, row, row + m->rows};
        chains.push_back(c);
        // after p passes the result sits in row (p even) or next (p odd)
        folds.push_back(SumDesc{(p % 2 == 0) ? row : row + m->rows, 0, m->rows, 0, row + 2 * m->rows});
        mo += (size_t)m->ld() * m->rows;
        vo += 2 * (size_t)m->rows + 1;
        nmax = std::max(nmax, m->rows);
        emax = std::max(emax, (long long)m->ld() * m->rows);
    }
    Batch<ChainDesc> bc = make_batch(ctx, chains);
    dim3 g0(blocks_for(emax, kThreads, std::max(1, 148 * 8 / (int)mats.size()) + 1), bc.count);
    if (cplx) moduli_kernel<true><<<g0, kThreads, 0, ctx.stream>>>(bc);
    else moduli_kernel<false><<<g0, kThreads, 0, ctx.stream>>>(bc);
    ctx.kernel_launches++;
    dim3 g1((nmax + 32 * kChainWarps - 1) / (32 * kChainWarps), bc.count);
    for (int step = 0; step < p; ++step) {
        abs_power_step_kernel<<<g1, 32 * kChainWarps, 0, ctx.stream>>>(bc, step & 1);
        ctx.kernel_launches++;
    }
    Batch<SumDesc> bf = make_batch(ctx, folds);
    max_fold_kernel<<<bf.count, 256, 0, ctx.stream>>>(bf);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
    std::vector<double> host(vec_total);
    TNS_CUDA(cudaMemcpyAsync(host.data(), vecs.p, sizeof(double) * vec_total, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    vo = 0;
    for (size_t k = 0; k < mats.size(); ++k) {
        out[k] = host[vo + 2 * (size_t)mats[k]->rows];
        vo += 2 * (size_t)mats[k]->rows + 1;
    }
    return out;
}

void panel_product_batch(Context& ctx, std::vector<PanelDesc>& v, bool cplx, bool adjoint) {
    if (v.empty()) return;
    int tmax = 0;
    for (auto& d : v) tmax = std::max(tmax, d.t);
    if (tmax > 16) fail(TNS_E_ARGUMENT, "internal panel product wider than 16 columns");
    if (cplx) {
        if (tmax <= 2) launch_panel<2, true>(ctx, v, adjoint);
        else if (tmax <= 4) launch_panel<4, true>(ctx, v, adjoint);
        else if (tmax <= 8) launch_panel<8, true>(ctx, v, adjoint);
        else launch_panel<16, true>(ctx, v, adjoint);
    } else {
        if (tmax <= 2) launch_panel<2, false>(ctx, v, adjoint);
        else if (tmax <= 4) launch_panel<4, false>(ctx, v, adjoint);
        else if (tmax <= 8) launch_panel<8, false>(ctx, v, adjoint);
        else launch_panel<16, false>(ctx, v, adjoint);
    }
}

// ---------------------------------------------------------------------------
// Single-matrix host entry points (one-item batches)
// ---------------------------------------------------------------------------

void scale_inplace(Context& ctx, void* c, int m, int n, int ldc, bool cplx, double br, double bi) {
    if (br == 1.0 && bi == 0.0) return;
    if ((long long)m * n == 0) return;
    scale_kernel<<<blocks_for((long long)m * n), kThreads, 0, ctx.stream>>>(static_cast<double*>(c), m, n, ldc, cplx, br, bi);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

void scale_detached(cudaStream_t stream, double* c, int m, int n, int ldc, bool cplx, double br, double bi) {
    if (br == 1.0 && bi == 0.0) return;
    if ((long long)m * n == 0) return;
    scale_kernel<<<blocks_for((long long)m * n), kThreads, 0, stream>>>(c, m, n, ldc, cplx, br, bi);
    TNS_CUDA(cudaGetLastError());
}

void scaled_copy(Context& ctx, DMat& dst, const DMat& src, double f) {
    std::vector<EwDesc> v{ew_scaled_copy(dst, src, f)};
    ew_batch(ctx, v);
}

void add_scaled(Context& ctx, DMat& t, const DMat& s, double f) {
    std::vector<EwDesc> v{ew_add_scaled(t, s, f)};
    ew_batch(ctx, v);
}

void set_identity(Context& ctx, DMat& dst, double f) {
    std::vector<EwDesc> v{ew_identity(dst, f)};
    ew_batch(ctx, v);
}

void pade_split(Context& ctx, DMat& den, DMat& num, const DMat& v, const DMat& u) {
    std::vector<EwDesc> d{ew_pade_split(den, num, v, u)};
    ew_batch(ctx, d);
}

double norm1(Context& ctx, const DMat& a) { return norm1_batch(ctx, {&a})[0]; }

double norminf(Context& ctx, const DMat& a) { return norminf_batch(ctx, {&a})[0]; }

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

double one_norm_abs_power(Context& ctx, const DMat& a, int p) { return abs_power_batch(ctx, {&a}, p)[0]; }

void panel_product(Context& ctx, const DMat& a, const double* x, int ldx, double* y, int ldy, int t, bool adjoint) {
    if (a.rows == 0 || t == 0) return;
    // Wider panels run as successive blocks of 16 columns; each column's
    // arithmetic is independent of the others.
    for (int c0 = 0; c0 < t; c0 += 16) {
        int tc = std::min(16, t - c0);
        size_t es = a.cplx ? 2 : 1;
        PanelDesc d{a.p, a.rows, a.ld(), x + (size_t)c0 * ldx * es, ldx, y + (size_t)c0 * ldy * es, ldy, tc};
        std::vector<PanelDesc> v{d};
        panel_product_batch(ctx, v, a.cplx, adjoint);
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
