// CPU oracle for the Tensile dense hot path -- TEST INFRASTRUCTURE ONLY.
//
// A restatement, in C++, of the reference library's CPU algorithms. Only the
// test suite, the smoke check and the benchmark's CPU-baseline leg may load
// this code; the CUDA library never does. Every function names the reference
// file:line it follows (paths relative to the reference project root).
//
// Floating point: compiled with -ffp-contract=off so that a*b+c is two
// roundings, as RyuJIT computes it. The only fused multiply-adds are the ones
// the reference writes explicitly: the GEMM micro-kernel's accumulate and its
// alpha write-back (src/Tensile.Kernels/MicroKernels.cs:82-142).
//
// Parity: partially pinned (see the header): pinned by the reference's known-
// answer tests and by scipy; the .NET Random / Array.Sort restatements are
// unverifiable without a .NET runtime.

#include "tensile_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <type_traits>
#include <utility>
#include <vector>

#include <immintrin.h>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ===========================================================================
// .NET seeded System.Random: the legacy subtractive generator (Knuth's
// ran3 as published in Numerical Recipes), which .NET keeps for seeded
// construction. Used for normest1's probe signs (src/Tensile/NormEstimate.cs:163,
// 304) and by the reference tests to build inputs.
// ===========================================================================
struct NetRandom {
    static constexpr int MBIG = 2147483647;
    static constexpr int MSEED = 161803398;
    int seed_array[56];
    int inext = 0, inextp = 21;

    explicit NetRandom(int seed) {
        int subtraction = (seed == std::numeric_limits<int>::min()) ? MBIG : std::abs(seed);
        int mj = MSEED - subtraction;
        seed_array[55] = mj;
        int mk = 1;
        for (int i = 1; i < 55; i++) {
            int ii = (21 * i) % 55;
            seed_array[ii] = mk;
            mk = mj - mk;
            if (mk < 0) mk += MBIG;
            mj = seed_array[ii];
        }
        for (int k = 1; k < 5; k++) {
            for (int i = 1; i < 56; i++) {
                seed_array[i] -= seed_array[1 + (i + 30) % 55];
                if (seed_array[i] < 0) seed_array[i] += MBIG;
            }
        }
        seed_array[0] = 0;
        inext = 0;
        inextp = 21;
    }

    int internal_sample() {
        int loc_next = inext, loc_nextp = inextp;
        if (++loc_next >= 56) loc_next = 1;
        if (++loc_nextp >= 56) loc_nextp = 1;
        int ret = seed_array[loc_next] - seed_array[loc_nextp];
        if (ret == MBIG) ret--;
        if (ret < 0) ret += MBIG;
        seed_array[loc_next] = ret;
        inext = loc_next;
        inextp = loc_nextp;
        return ret;
    }

    double sample() { return internal_sample() * (1.0 / MBIG); }
    int next(int max_value) { return (int)(sample() * max_value); }
};

// ===========================================================================
// .NET Array.Sort(double[] keys, int[] items) with the default comparer:
// NaNs moved to the front, then introsort (insertion sort at <= 16, heapsort
// past the depth limit, median-of-three partition). Unstable on ties, so the
// tie order of normest1's candidate list (src/Tensile/NormEstimate.cs:380)
// follows exactly this sequence of swaps.
// ===========================================================================
struct NetSort {
    double* k;
    int* v;

    void swap(int i, int j) {
        std::swap(k[i], k[j]);
        std::swap(v[i], v[j]);
    }
    void swap_if_greater(int i, int j) {
        if (k[i] > k[j]) swap(i, j);
    }
    void insertion(int lo, int len) {
        for (int i = 0; i < len - 1; i++) {
            double t = k[lo + i + 1];
            int tv = v[lo + i + 1];
            int j = i;
            while (j >= 0 && t < k[lo + j]) {
                k[lo + j + 1] = k[lo + j];
                v[lo + j + 1] = v[lo + j];
                j--;
            }
            k[lo + j + 1] = t;
            v[lo + j + 1] = tv;
        }
    }
    void down_heap(int lo, int i, int n) {
        double d = k[lo + i - 1];
        int dv = v[lo + i - 1];
        while (i <= (n >> 1)) {
            int child = 2 * i;
            if (child < n && k[lo + child - 1] < k[lo + child]) child++;
            if (!(d < k[lo + child - 1])) break;
            k[lo + i - 1] = k[lo + child - 1];
            v[lo + i - 1] = v[lo + child - 1];
            i = child;
        }
        k[lo + i - 1] = d;
        v[lo + i - 1] = dv;
    }
    void heap(int lo, int n) {
        for (int i = n >> 1; i >= 1; i--) down_heap(lo, i, n);
        for (int i = n; i > 1; i--) {
            swap(lo, lo + i - 1);
            down_heap(lo, 1, i - 1);
        }
    }
    int partition(int lo, int len) {
        int hi = len - 1;
        int middle = hi >> 1;
        swap_if_greater(lo, lo + middle);
        swap_if_greater(lo, lo + hi);
        swap_if_greater(lo + middle, lo + hi);
        double pivot = k[lo + middle];
        swap(lo + middle, lo + hi - 1);
        int left = 0, right = hi - 1;
        while (left < right) {
            while (pivot > k[lo + (++left)]) {}
            while (pivot < k[lo + (--right)]) {}
            if (left >= right) break;
            swap(lo + left, lo + right);
        }
        if (left != hi - 1) swap(lo + left, lo + hi - 1);
        return left;
    }
    void intro(int lo, int len, int depth) {
        int size = len;
        while (size > 1) {
            if (size <= 16) {
                if (size == 2) {
                    swap_if_greater(lo, lo + 1);
                    return;
                }
                if (size == 3) {
                    swap_if_greater(lo, lo + 1);
                    swap_if_greater(lo, lo + 2);
                    swap_if_greater(lo + 1, lo + 2);
                    return;
                }
                insertion(lo, size);
                return;
            }
            if (depth == 0) {
                heap(lo, size);
                return;
            }
            depth--;
            int p = partition(lo, size);
            intro(lo + p + 1, size - (p + 1), depth);
            size = p;
        }
    }
    static int floor_log2(unsigned x) {
        int r = 0;
        while (x >>= 1) r++;
        return r;
    }
    void sort(int n) {
        if (n <= 1) return;
        int left = 0;
        for (int i = 0; i < n; i++) {
            if (std::isnan(k[i])) {
                std::swap(k[left], k[i]);
                std::swap(v[left], v[i]);
                left++;
            }
        }
        if (left == n) return;
        NetSort rest{k + left, v + left};
        int len = n - left;
        rest.intro(0, len, 2 * (floor_log2((unsigned)len) + 1));
    }
};

// ===========================================================================
// System.Numerics.Complex arithmetic, as .NET publishes it.
// ===========================================================================
struct cplx {
    double re, im;
};
inline bool operator==(cplx a, cplx b) { return a.re == b.re && a.im == b.im; }
inline cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
inline cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
inline cplx cneg(cplx a) { return {-a.re, -a.im}; }
// (a+bi)(c+di) = (ac - bd) + (bc + ad)i
inline cplx cmul(cplx a, cplx b) {
    return {(a.re * b.re) - (a.im * b.im), (a.im * b.re) + (a.re * b.im)};
}
// Smith's division.
inline cplx cdiv(cplx l, cplx r) {
    double a = l.re, b = l.im, c = r.re, d = r.im;
    if (std::fabs(d) < std::fabs(c)) {
        double doc = d / c;
        return {(a + b * doc) / (c + d * doc), (b - a * doc) / (c + d * doc)};
    }
    double cod = c / d;
    return {(b + a * cod) / (d + c * cod), (-a + b * cod) / (d + c * cod)};
}
// Complex.Abs: scaled hypot.
inline double cabs_net(cplx z) {
    double a = std::fabs(z.re), b = std::fabs(z.im);
    double small, large;
    if (a < b) {
        small = a;
        large = b;
    } else {
        small = b;
        large = a;
    }
    if (small == 0.0) return large;
    if (std::isinf(large) && !std::isnan(small)) return std::numeric_limits<double>::infinity();
    double ratio = small / large;
    return large * std::sqrt(1.0 + ratio * ratio);
}
inline cplx cexp_net(cplx z) {
    double e = std::exp(z.re);
    return {e * std::cos(z.im), e * std::sin(z.im)};
}
inline cplx cconj(cplx z) { return {z.re, -z.im}; }
inline cplx operator-(cplx a) { return cneg(a); }

// Math.Max / Math.Min as .NET Core implements them (IEEE 754:2019 maximum /
// minimum: NaN propagates, +0 beats -0).
inline double net_max(double a, double b) {
    if (a != b) {
        if (!std::isnan(a)) return b < a ? a : b;
        return a;
    }
    return std::signbit(b) ? a : b;
}
inline double net_min(double a, double b) {
    if (a != b) {
        if (!std::isnan(a)) return a < b ? a : b;
        return a;
    }
    return std::signbit(a) ? a : b;
}

int g_threads = 0;
int threads_now() {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

// ===========================================================================
// Real GEMM with the reference's blocking semantics.
// src/Tensile.Kernels/Gemm.cs:117-203 (serial, KC=384),
// src/Tensile.Kernels/ParallelGemm.cs:138-229 (threaded, KC=256, work >= 2^24,
// src/Tensile.Kernels/GemmDispatch.cs:45,109), micro-kernels
// src/Tensile.Kernels/MicroKernels.cs:57-273. Every C element is computed as
// c = beta-scaled C, then per KC slab: acc = sum of fma(a, b, acc) in k order,
// c = fma(alpha, acc, c). That is independent of MR/NR and of the thread split,
// so the micro-kernel geometry here (8x6) gives the same bits as the
// reference's 16x8 and 8x6 kernels for alpha = +-1.
// ===========================================================================
constexpr int MR = 8, NR = 6, MC = 144, NC = 4096;

// The 8x6 AVX2/FMA register tile (the reference's Avx2Kernel8x6 geometry):
// 12 accumulators, each lane a k-ordered fused multiply-add chain.
inline void micro_kernel(int kc, double alpha, const double* ap, const double* bp, double* c,
                         int ldc, int mrb, int nrb) {
    __m256d c00 = _mm256_setzero_pd(), c10 = _mm256_setzero_pd();
    __m256d c01 = _mm256_setzero_pd(), c11 = _mm256_setzero_pd();
    __m256d c02 = _mm256_setzero_pd(), c12 = _mm256_setzero_pd();
    __m256d c03 = _mm256_setzero_pd(), c13 = _mm256_setzero_pd();
    __m256d c04 = _mm256_setzero_pd(), c14 = _mm256_setzero_pd();
    __m256d c05 = _mm256_setzero_pd(), c15 = _mm256_setzero_pd();
    for (int p = 0; p < kc; p++) {
        __m256d a0 = _mm256_loadu_pd(ap);
        __m256d a1 = _mm256_loadu_pd(ap + 4);
        ap += MR;
        __m256d b;
        b = _mm256_broadcast_sd(bp + 0);
        c00 = _mm256_fmadd_pd(a0, b, c00);
        c10 = _mm256_fmadd_pd(a1, b, c10);
        b = _mm256_broadcast_sd(bp + 1);
        c01 = _mm256_fmadd_pd(a0, b, c01);
        c11 = _mm256_fmadd_pd(a1, b, c11);
        b = _mm256_broadcast_sd(bp + 2);
        c02 = _mm256_fmadd_pd(a0, b, c02);
        c12 = _mm256_fmadd_pd(a1, b, c12);
        b = _mm256_broadcast_sd(bp + 3);
        c03 = _mm256_fmadd_pd(a0, b, c03);
        c13 = _mm256_fmadd_pd(a1, b, c13);
        b = _mm256_broadcast_sd(bp + 4);
        c04 = _mm256_fmadd_pd(a0, b, c04);
        c14 = _mm256_fmadd_pd(a1, b, c14);
        b = _mm256_broadcast_sd(bp + 5);
        c05 = _mm256_fmadd_pd(a0, b, c05);
        c15 = _mm256_fmadd_pd(a1, b, c15);
        bp += NR;
    }
    __m256d lo[NR] = {c00, c01, c02, c03, c04, c05};
    __m256d hi[NR] = {c10, c11, c12, c13, c14, c15};
    __m256d va = _mm256_set1_pd(alpha);
    if (mrb == MR && nrb == NR) {
        for (int j = 0; j < NR; j++) {
            double* col = c + (size_t)j * ldc;
            _mm256_storeu_pd(col, _mm256_fmadd_pd(va, lo[j], _mm256_loadu_pd(col)));
            _mm256_storeu_pd(col + 4, _mm256_fmadd_pd(va, hi[j], _mm256_loadu_pd(col + 4)));
        }
        return;
    }
    alignas(32) double acc[NR][MR];
    for (int j = 0; j < NR; j++) {
        _mm256_store_pd(&acc[j][0], lo[j]);
        _mm256_store_pd(&acc[j][4], hi[j]);
    }
    for (int j = 0; j < nrb; j++) {
        double* col = c + (size_t)j * ldc;
        for (int i = 0; i < mrb; i++) col[i] = __builtin_fma(alpha, acc[j][i], col[i]);
    }
}

void pack_a(int m, int kc, const double* a, int lda, double* ap) {
    int panels = (m + MR - 1) / MR;
    for (int q = 0; q < panels; q++) {
        int i0 = q * MR, rows = std::min(MR, m - i0);
        double* dst = ap + (size_t)q * MR * kc;
        for (int p = 0; p < kc; p++) {
            const double* src = a + (size_t)p * lda + i0;
            for (int i = 0; i < rows; i++) dst[p * MR + i] = src[i];
            for (int i = rows; i < MR; i++) dst[p * MR + i] = 0.0;
        }
    }
}

void pack_b_panel(int kc, int cols, const double* b, int ldb, double* bp) {
    for (int p = 0; p < kc; p++) {
        for (int j = 0; j < cols; j++) bp[p * NR + j] = b[(size_t)j * ldb + p];
        for (int j = cols; j < NR; j++) bp[p * NR + j] = 0.0;
    }
}

void scale_c(int m, int n, double beta, double* c, int ldc) {
    if (beta == 1.0) return;
    for (int j = 0; j < n; j++) {
        double* col = c + (size_t)j * ldc;
        if (beta == 0.0)
            std::memset(col, 0, sizeof(double) * (size_t)m);
        else
            for (int i = 0; i < m; i++) col[i] *= beta;
    }
}

void dgemm_impl(int m, int n, int k, double alpha, const double* a, int lda, const double* b,
                int ldb, double beta, double* c, int ldc, bool multithreaded) {
    if (m <= 0 || n <= 0) return;
    scale_c(m, n, beta, c, ldc);
    if (k == 0 || alpha == 0.0) return;
    bool threaded = multithreaded && (int64_t)m * n * k >= (int64_t)1 << 24;
    int kcmax = threaded ? 256 : 384;
    int nthreads = threaded ? threads_now() : 1;
    int a_panels = (m + MR - 1) / MR;
    std::vector<double> ap((size_t)a_panels * MR * kcmax);
    for (int jc = 0; jc < n; jc += NC) {
        int nc = std::min(NC, n - jc);
        int b_panels = (nc + NR - 1) / NR;
        std::vector<double> bp((size_t)b_panels * NR * kcmax);
        for (int pc = 0; pc < k; pc += kcmax) {
            int kc = std::min(kcmax, k - pc);
#pragma omp parallel for num_threads(nthreads) schedule(static) if (nthreads > 1)
            for (int q = 0; q < b_panels; q++) {
                int cols = std::min(NR, nc - q * NR);
                pack_b_panel(kc, cols, b + (size_t)(jc + q * NR) * ldb + pc, ldb,
                             bp.data() + (size_t)q * NR * kc);
            }
#pragma omp parallel for num_threads(nthreads) schedule(static) if (nthreads > 1)
            for (int q = 0; q < a_panels; q++) {
                int rows = std::min(MR, m - q * MR);
                pack_a(rows, kc, a + (size_t)pc * lda + q * MR, lda, ap.data() + (size_t)q * MR * kc);
            }
            for (int ic = 0; ic < m; ic += MC) {
                int mc = std::min(MC, m - ic);
                int first = ic / MR, count = (mc + MR - 1) / MR;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic) if (nthreads > 1)
                for (int q = 0; q < b_panels; q++) {
                    int nrb = std::min(NR, nc - q * NR);
                    const double* bpan = bp.data() + (size_t)q * NR * kc;
                    for (int t = 0; t < count; t++) {
                        int ir = t * MR;
                        int mrb = std::min(MR, mc - ir);
                        micro_kernel(kc, alpha, ap.data() + (size_t)(first + t) * MR * kc, bpan,
                                     c + (size_t)(jc + q * NR) * ldc + ic + ir, ldc, mrb, nrb);
                    }
                }
            }
        }
    }
}

// ===========================================================================
// Complex 4M product. src/Tensile/ComplexKernels.cs:49-108 (four real GEMMs,
// never 3M), Split :187-201, Combine :213-240.
// ===========================================================================
void split(int m, int n, const cplx* s, int lds, double* re, double* im) {
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            cplx z = s[(size_t)j * lds + i];
            re[(size_t)j * m + i] = z.re;
            im[(size_t)j * m + i] = z.im;
        }
}

void zgemm_impl(int m, int n, int k, cplx alpha, const cplx* a, int lda, const cplx* b, int ldb,
                cplx beta, cplx* c, int ldc, bool mt) {
    if (m <= 0 || n <= 0) return;
    std::vector<double> ar((size_t)m * k), ai((size_t)m * k), br((size_t)k * n), bi((size_t)k * n);
    std::vector<double> pr((size_t)m * n), pi((size_t)m * n);
    split(m, k, a, lda, ar.data(), ai.data());
    split(k, n, b, ldb, br.data(), bi.data());
    int lk = std::max(k, 1), lm = std::max(m, 1);
    dgemm_impl(m, n, k, 1.0, ar.data(), lm, br.data(), lk, 0.0, pr.data(), lm, mt);
    dgemm_impl(m, n, k, -1.0, ai.data(), lm, bi.data(), lk, 1.0, pr.data(), lm, mt);
    dgemm_impl(m, n, k, 1.0, ar.data(), lm, bi.data(), lk, 0.0, pi.data(), lm, mt);
    dgemm_impl(m, n, k, 1.0, ai.data(), lm, br.data(), lk, 1.0, pi.data(), lm, mt);
    bool unit_alpha = alpha == cplx{1.0, 0.0};
    bool real_alpha = alpha.im == 0.0;
    bool zero_beta = beta == cplx{0.0, 0.0};
    bool unit_beta = beta == cplx{1.0, 0.0};
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            double p = pr[(size_t)j * m + i], q = pi[(size_t)j * m + i];
            cplx prod = unit_alpha  ? cplx{p, q}
                        : real_alpha ? cplx{alpha.re * p, alpha.re * q}
                                     : cmul(alpha, cplx{p, q});
            cplx& t = c[(size_t)j * ldc + i];
            t = zero_beta ? prod : unit_beta ? cadd(t, prod) : cadd(cmul(beta, t), prod);
        }
}

// ===========================================================================
// Streaming column operations. src/Tensile.Kernels/ColumnOps.cs:35-108.
// Vector<double> is 256-bit (4 lanes) under .NET's defaults; the dot keeps its
// four vector accumulators and the lane sum (e0+e1)+(e2+e3).
// ===========================================================================
constexpr int W = 4;

double col_dot(int n, const double* x, const double* y) {
    int i = 0;
    double total = 0.0;
    if (n >= W) {
        double a0[W] = {0}, a1[W] = {0}, a2[W] = {0}, a3[W] = {0};
        for (; i <= n - 4 * W; i += 4 * W)
            for (int l = 0; l < W; l++) {
                a0[l] = a0[l] + x[i + l] * y[i + l];
                a1[l] = a1[l] + x[i + W + l] * y[i + W + l];
                a2[l] = a2[l] + x[i + 2 * W + l] * y[i + 2 * W + l];
                a3[l] = a3[l] + x[i + 3 * W + l] * y[i + 3 * W + l];
            }
        for (; i <= n - W; i += W)
            for (int l = 0; l < W; l++) a0[l] = a0[l] + x[i + l] * y[i + l];
        double s[W];
        for (int l = 0; l < W; l++) s[l] = (a0[l] + a1[l]) + (a2[l] + a3[l]);
        total = (s[0] + s[1]) + (s[2] + s[3]);
    }
    for (; i < n; i++) total += x[i] * y[i];
    return total;
}
inline void col_axpy(int n, double alpha, const double* x, double* y) {
    for (int i = 0; i < n; i++) y[i] = y[i] + alpha * x[i];
}
inline void col_scale(int n, double alpha, double* x) {
    for (int i = 0; i < n; i++) x[i] *= alpha;
}

// src/Tensile.Kernels/Pivoting.cs:25-89: first index of the largest |x|,
// with the four-lane scan's NaN behaviour.
int index_of_max_abs(int n, const double* x) {
    if (n <= 0) return 0;
    int best = 0;
    double best_value = std::fabs(x[0]);
    int i = 1;
    if (n >= 2 * W) {
        double bv[W];
        long bi[W];
        for (int l = 0; l < W; l++) {
            bv[l] = std::fabs(x[l]);
            bi[l] = l;
        }
        for (i = W; i <= n - W; i += W)
            for (int l = 0; l < W; l++) {
                double v = std::fabs(x[i + l]);
                if (v > bv[l]) {
                    bv[l] = v;
                    bi[l] = i + l;
                }
            }
        best_value = bv[0];
        best = (int)bi[0];
        for (int l = 1; l < W; l++) {
            double v = bv[l];
            int idx = (int)bi[l];
            if (v > best_value || (v == best_value && idx < best)) {
                best_value = v;
                best = idx;
            }
        }
    }
    for (; i < n; i++) {
        double v = std::fabs(x[i]);
        if (v > best_value) {
            best_value = v;
            best = i;
        }
    }
    return best;
}

// ===========================================================================
// Real triangular solves. src/Tensile.Kernels/Triangular.cs:26-228.
// ===========================================================================
void update_four(int n, const double* x, double* c0, double* c1, double* c2, double* c3,
                 double v0, double v1, double v2, double v3) {
    double a0 = -v0, a1 = -v1, a2 = -v2, a3 = -v3;
    for (int i = 0; i < n; i++) {
        double xv = x[i];
        c0[i] = c0[i] + a0 * xv;
        c1[i] = c1[i] + a1 * xv;
        c2[i] = c2[i] + a2 * xv;
        c3[i] = c3[i] + a3 * xv;
    }
}

void solve_lower_unit(int m, int n, const double* l, int ldl, double* b, int ldb) {
    int j = 0;
    for (; j + 4 <= n; j += 4) {
        double *c0 = b + (size_t)j * ldb, *c1 = c0 + ldb, *c2 = c1 + ldb, *c3 = c2 + ldb;
        for (int p = 0; p < m - 1; p++) {
            double v0 = c0[p], v1 = c1[p], v2 = c2[p], v3 = c3[p];
            if (v0 == 0.0 && v1 == 0.0 && v2 == 0.0 && v3 == 0.0) continue;
            update_four(m - p - 1, l + (size_t)p * ldl + p + 1, c0 + p + 1, c1 + p + 1, c2 + p + 1,
                        c3 + p + 1, v0, v1, v2, v3);
        }
    }
    for (; j < n; j++) {
        double* col = b + (size_t)j * ldb;
        for (int p = 0; p < m - 1; p++) {
            double v = col[p];
            if (v != 0.0) col_axpy(m - p - 1, -v, l + (size_t)p * ldl + p + 1, col + p + 1);
        }
    }
}

void solve_upper(int m, int n, const double* u, int ldu, double* b, int ldb) {
    int j = 0;
    for (; j + 4 <= n; j += 4) {
        double *c0 = b + (size_t)j * ldb, *c1 = c0 + ldb, *c2 = c1 + ldb, *c3 = c2 + ldb;
        for (int p = m - 1; p >= 0; p--) {
            double d = u[(size_t)p * ldu + p];
            c0[p] /= d;
            c1[p] /= d;
            c2[p] /= d;
            c3[p] /= d;
            double v0 = c0[p], v1 = c1[p], v2 = c2[p], v3 = c3[p];
            if (p == 0 || (v0 == 0.0 && v1 == 0.0 && v2 == 0.0 && v3 == 0.0)) continue;
            update_four(p, u + (size_t)p * ldu, c0, c1, c2, c3, v0, v1, v2, v3);
        }
    }
    for (; j < n; j++) {
        double* col = b + (size_t)j * ldb;
        for (int p = m - 1; p >= 0; p--) {
            col[p] /= u[(size_t)p * ldu + p];
            double v = col[p];
            if (v != 0.0 && p > 0) col_axpy(p, -v, u + (size_t)p * ldu, col);
        }
    }
}

void solve_upper_transposed(int m, int n, const double* u, int ldu, double* b, int ldb) {
    for (int j = 0; j < n; j++) {
        double* col = b + (size_t)j * ldb;
        for (int i = 0; i < m; i++) {
            const double* ui = u + (size_t)i * ldu;
            col[i] = (col[i] - col_dot(i, ui, col)) / ui[i];
        }
    }
}

// src/Tensile.Kernels/Triangular.cs:131-150: explicit diagonal, one column at a time.
void solve_lower(int m, int n, const double* l, int ldl, double* b, int ldb) {
    for (int j = 0; j < n; j++) {
        double* col = b + (size_t)j * ldb;
        for (int p = 0; p < m; p++) {
            const double* lp = l + (size_t)p * ldl;
            col[p] /= lp[p];
            double v = col[p];
            if (v != 0.0 && p + 1 < m) col_axpy(m - p - 1, -v, lp + p + 1, col + p + 1);
        }
    }
}

// src/Tensile.Kernels/Triangular.cs:157-168.
void solve_lower_transposed(int m, int n, const double* l, int ldl, double* b, int ldb) {
    for (int j = 0; j < n; j++) {
        double* col = b + (size_t)j * ldb;
        for (int i = m - 1; i >= 0; i--) {
            const double* li = l + (size_t)i * ldl;
            col[i] = (col[i] - col_dot(m - i - 1, li + i + 1, col + i + 1)) / li[i];
        }
    }
}

void solve_lower_unit_transposed(int m, int n, const double* l, int ldl, double* b, int ldb) {
    for (int j = 0; j < n; j++) {
        double* col = b + (size_t)j * ldb;
        for (int i = m - 1; i >= 0; i--) {
            const double* li = l + (size_t)i * ldl;
            col[i] -= col_dot(m - i - 1, li + i + 1, col + i + 1);
        }
    }
}

template <typename T>
void swap_rows(T* a, int lda, int c0, int c1, const int* piv, int first, int last) {
    for (int j = c0; j < c1; j++) {
        T* col = a + (size_t)j * lda;
        for (int k = first; k < last; k++) {
            int p = piv[k];
            if (p != k) std::swap(col[k], col[p]);
        }
    }
}
template <typename T>
void unswap_rows(T* a, int lda, int c0, int c1, const int* piv, int first, int last) {
    for (int j = c0; j < c1; j++) {
        T* col = a + (size_t)j * lda;
        for (int k = last - 1; k >= first; k--) {
            int p = piv[k];
            if (p != k) std::swap(col[k], col[p]);
        }
    }
}

constexpr double SafeMin = 2.2250738585072014e-308;

int default_block_size(int m, int n) { return std::min(m, n) < 1024 ? 32 : 64; }

// src/Tensile.Kernels/Lu.cs:384-424
void factor_panel_real(int m, int n, double* a, int lda, int* piv, int offset, orc_lu_info* info) {
    int limit = std::min(m, n);
    for (int j = 0; j < limit; j++) {
        double* col = a + (size_t)j * lda;
        int p = j + index_of_max_abs(m - j, col + j);
        piv[j] = p;
        double value = col[p];
        if (value == 0.0) {
            if (info->singular_column < 0) info->singular_column = offset + j;
        } else {
            if (p != j)
                for (int jj = 0; jj < n; jj++) std::swap(a[(size_t)jj * lda + j], a[(size_t)jj * lda + p]);
            if (std::fabs(value) >= SafeMin)
                col_scale(m - j - 1, 1.0 / value, col + j + 1);
            else
                for (int i = j + 1; i < m; i++) col[i] /= value;
        }
        for (int jj = j + 1; jj < n; jj++) {
            double* target = a + (size_t)jj * lda;
            double mult = target[j];
            if (mult != 0.0) col_axpy(m - j - 1, -mult, col + j + 1, target + j + 1);
        }
    }
}

// src/Tensile.Kernels/Lu.cs:230-329 (Factor, RecordPivotRange)
void dgetrf_impl(int m, int n, double* a, int lda, int nb, int* piv, orc_lu_info* info) {
    info->singular_column = -1;
    info->smallest_pivot = 0.0;
    info->largest_pivot = 0.0;
    int limit = std::min(m, n);
    if (limit == 0) return;
    if (nb < 1) nb = default_block_size(m, n);
    if (nb >= limit) {
        factor_panel_real(m, n, a, lda, piv, 0, info);
    } else {
        for (int jb = 0; jb < limit; jb += nb) {
            int w = std::min(nb, limit - jb);
            factor_panel_real(m - jb, w, a + (size_t)jb * lda + jb, lda, piv + jb, jb, info);
            for (int i = 0; i < w; i++) piv[jb + i] += jb;
            swap_rows(a, lda, 0, jb, piv, jb, jb + w);
            if (jb + w >= n) continue;
            swap_rows(a, lda, jb + w, n, piv, jb, jb + w);
            solve_lower_unit(w, n - jb - w, a + (size_t)jb * lda + jb, lda,
                             a + (size_t)(jb + w) * lda + jb, lda);
            if (jb + w >= m) continue;
            dgemm_impl(m - jb - w, n - jb - w, w, -1.0, a + (size_t)jb * lda + jb + w, lda,
                       a + (size_t)(jb + w) * lda + jb, lda, 1.0,
                       a + (size_t)(jb + w) * lda + jb + w, lda, true);
        }
    }
    double smallest = std::numeric_limits<double>::infinity(), largest = 0.0;
    for (int j = 0; j < limit; j++) {
        double v = std::fabs(a[(size_t)j * lda + j]);
        smallest = net_min(smallest, v);
        largest = net_max(largest, v);
    }
    info->smallest_pivot = smallest;
    info->largest_pivot = largest;
}

// ===========================================================================
// Complex (generic) LU. src/Tensile/BlockedLu.cs:45-413.
// ===========================================================================
inline double pivot_magnitude(cplx z) { return std::fabs(z.re) + std::fabs(z.im); }

int index_of_largest_pivot(int n, const cplx* x) {
    if (n <= 0) return 0;
    int best = 0;
    double bv = pivot_magnitude(x[0]);
    for (int i = 1; i < n; i++) {
        double v = pivot_magnitude(x[i]);
        if (v > bv) {
            bv = v;
            best = i;
        }
    }
    return best;
}

void factor_panel_complex(int m, int n, cplx* a, int lda, int* piv, int offset, orc_lu_info* info) {
    int limit = std::min(m, n);
    const cplx zero{0.0, 0.0};
    for (int j = 0; j < limit; j++) {
        cplx* col = a + (size_t)j * lda;
        int p = j + index_of_largest_pivot(m - j, col + j);
        piv[j] = p;
        cplx value = col[p];
        if (value == zero) {
            if (info->singular_column < 0) info->singular_column = offset + j;
        } else {
            if (p != j)
                for (int jj = 0; jj < n; jj++) std::swap(a[(size_t)jj * lda + j], a[(size_t)jj * lda + p]);
            if (cabs_net(value) >= SafeMin) {
                cplx r = cdiv(cplx{1.0, 0.0}, value);
                for (int i = j + 1; i < m; i++) col[i] = cmul(col[i], r);
            } else {
                for (int i = j + 1; i < m; i++) col[i] = cdiv(col[i], value);
            }
        }
        for (int jj = j + 1; jj < n; jj++) {
            cplx* target = a + (size_t)jj * lda;
            cplx mult = target[j];
            if (mult == zero) continue;
            cplx scale = cneg(mult);
            for (int i = j + 1; i < m; i++) target[i] = cadd(target[i], cmul(scale, col[i]));
        }
    }
}

// src/Tensile/BlockedLu.cs:312-327 (the generic unit-lower solve)
void zsolve_lower_unit(int n, int ncols, const cplx* l, int ldl, cplx* b, int ldb) {
    const cplx zero{0.0, 0.0};
    for (int c = 0; c < ncols; c++) {
        cplx* x = b + (size_t)c * ldb;
        for (int k = 0; k < n; k++) {
            cplx xk = x[k];
            if (xk == zero) continue;
            cplx scale = cneg(xk);
            const cplx* below = l + (size_t)k * ldl;
            for (int i = k + 1; i < n; i++) x[i] = cadd(x[i], cmul(scale, below[i]));
        }
    }
}

void zsolve_upper(int n, int ncols, const cplx* u, int ldu, cplx* b, int ldb) {
    const cplx zero{0.0, 0.0};
    for (int c = 0; c < ncols; c++) {
        cplx* x = b + (size_t)c * ldb;
        for (int k = n - 1; k >= 0; k--) {
            const cplx* col = u + (size_t)k * ldu;
            if (x[k] == zero) continue;
            x[k] = cdiv(x[k], col[k]);
            cplx scale = cneg(x[k]);
            for (int i = 0; i < k; i++) x[i] = cadd(x[i], cmul(scale, col[i]));
        }
    }
}

void zsolve_upper_adjoint(int n, int ncols, const cplx* u, int ldu, cplx* b, int ldb) {
    for (int c = 0; c < ncols; c++) {
        cplx* x = b + (size_t)c * ldb;
        for (int i = 0; i < n; i++) {
            const cplx* col = u + (size_t)i * ldu;
            cplx sum = x[i];
            for (int k = 0; k < i; k++) sum = csub(sum, cmul(cconj(col[k]), x[k]));
            x[i] = cdiv(sum, cconj(col[i]));
        }
    }
}

void zsolve_lower_unit_adjoint(int n, int ncols, const cplx* l, int ldl, cplx* b, int ldb) {
    for (int c = 0; c < ncols; c++) {
        cplx* x = b + (size_t)c * ldb;
        for (int i = n - 1; i >= 0; i--) {
            const cplx* col = l + (size_t)i * ldl;
            cplx sum = x[i];
            for (int k = i + 1; k < n; k++) sum = csub(sum, cmul(cconj(col[k]), x[k]));
            x[i] = sum;
        }
    }
}

void zgetrf_impl(int m, int n, cplx* a, int lda, int nb, int* piv, orc_lu_info* info) {
    info->singular_column = -1;
    info->smallest_pivot = 0.0;
    info->largest_pivot = 0.0;
    int limit = std::min(m, n);
    if (limit == 0) return;
    if (nb < 1) nb = default_block_size(m, n);
    if (nb >= limit) {
        factor_panel_complex(m, n, a, lda, piv, 0, info);
    } else {
        for (int jb = 0; jb < limit; jb += nb) {
            int w = std::min(nb, limit - jb);
            factor_panel_complex(m - jb, w, a + (size_t)jb * lda + jb, lda, piv + jb, jb, info);
            for (int i = 0; i < w; i++) piv[jb + i] += jb;
            swap_rows(a, lda, 0, jb, piv, jb, jb + w);
            if (jb + w >= n) continue;
            swap_rows(a, lda, jb + w, n, piv, jb, jb + w);
            zsolve_lower_unit(w, n - jb - w, a + (size_t)jb * lda + jb, lda,
                              a + (size_t)(jb + w) * lda + jb, lda);
            if (jb + w >= m) continue;
            zgemm_impl(m - jb - w, n - jb - w, w, cplx{-1.0, 0.0}, a + (size_t)jb * lda + jb + w, lda,
                       a + (size_t)(jb + w) * lda + jb, lda, cplx{1.0, 0.0},
                       a + (size_t)(jb + w) * lda + jb + w, lda, true);
        }
    }
    double smallest = std::numeric_limits<double>::infinity(), largest = 0.0;
    for (int j = 0; j < limit; j++) {
        double v = cabs_net(a[(size_t)j * lda + j]);
        smallest = net_min(smallest, v);
        largest = net_max(largest, v);
    }
    info->smallest_pivot = smallest;
    info->largest_pivot = largest;
}

// ===========================================================================
// Element-type traits: the reference's IElementKernels<T>
// (src/Tensile/ElementKernels.cs:46-170, src/Tensile/ComplexKernels.cs:110-180).
// ===========================================================================
double one_norm_real(int m, int n, const double* a, int lda) {
    double best = 0.0;
    for (int j = 0; j < n; j++) {
        const double* col = a + (size_t)j * lda;
        double sum = 0.0;
        for (int i = 0; i < m; i++) sum += std::fabs(col[i]);
        best = net_max(best, sum);
    }
    return best;
}
double inf_norm_real(int m, int n, const double* a, int lda) {
    if (m == 0 || n == 0) return 0.0;
    std::vector<double> sums(m, 0.0);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) sums[i] += std::fabs(a[(size_t)j * lda + i]);
    double best = 0.0;
    for (int i = 0; i < m; i++) best = net_max(best, sums[i]);
    return best;
}
double one_norm_complex(int m, int n, const cplx* a, int lda) {
    if (m == 0 || n == 0) return 0.0;
    double best = 0.0;
    for (int j = 0; j < n; j++) {
        double sum = 0.0;
        for (int i = 0; i < m; i++) sum += cabs_net(a[(size_t)j * lda + i]);
        best = net_max(best, sum);
    }
    return best;
}
double inf_norm_complex(int m, int n, const cplx* a, int lda) {
    if (m == 0 || n == 0) return 0.0;
    std::vector<double> sums(m, 0.0);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) sums[i] += cabs_net(a[(size_t)j * lda + i]);
    double best = 0.0;
    for (int i = 0; i < m; i++) best = net_max(best, sums[i]);
    return best;
}

struct RealK {
    using T = double;
    static constexpr bool discrete = true;
    static T one() { return 1.0; }
    static T zero() { return 0.0; }
    static T neg(T x) { return -x; }
    static double magnitude(T x) { return std::fabs(x); }
    static T sign(T x) { return x >= 0.0 ? 1.0 : -1.0; }
    static T scale(T x, double f) { return x * f; }
    static T mul(T a, T b) { return a * b; }
    static T add(T a, T b) { return a + b; }
    static T div_real(T a, double d) { return a / d; }
    static T exp(T x) { return std::exp(x); }
    static bool eq(T a, T b) { return a == b; }
    static double one_norm(int m, int n, const T* a, int lda) { return one_norm_real(m, n, a, lda); }
    static double inf_norm(int m, int n, const T* a, int lda) { return inf_norm_real(m, n, a, lda); }
    static void gemm(int m, int n, int k, const T* a, int lda, const T* b, int ldb, T beta, T* c,
                     int ldc) {
        dgemm_impl(m, n, k, 1.0, a, lda, b, ldb, beta, c, ldc, true);
    }
};

struct ComplexK {
    using T = cplx;
    static constexpr bool discrete = false;
    static T one() { return {1.0, 0.0}; }
    static T zero() { return {0.0, 0.0}; }
    static T neg(T x) { return cneg(x); }
    static double magnitude(T x) { return cabs_net(x); }
    static T sign(T x) {
        if (x == T{0.0, 0.0}) return {1.0, 0.0};
        double mod = cabs_net(x);
        return {x.re / mod, x.im / mod};
    }
    static T scale(T x, double f) { return {x.re * f, x.im * f}; }
    static T mul(T a, T b) { return cmul(a, b); }
    static T add(T a, T b) { return cadd(a, b); }
    static T div_real(T a, double d) { return cdiv(a, cplx{d, 0.0}); }
    static T exp(T x) { return cexp_net(x); }
    static bool eq(T a, T b) { return a == b; }
    static double one_norm(int m, int n, const T* a, int lda) { return one_norm_complex(m, n, a, lda); }
    static double inf_norm(int m, int n, const T* a, int lda) { return inf_norm_complex(m, n, a, lda); }
    static void gemm(int m, int n, int k, const T* a, int lda, const T* b, int ldb, T beta, T* c,
                     int ldc) {
        zgemm_impl(m, n, k, cplx{1.0, 0.0}, a, lda, b, ldb, beta, c, ldc, true);
    }
};

// ===========================================================================
// Operators. src/Tensile/LinearOperators.cs:89-350,
// src/Tensile.Kernels/PanelProduct.cs:25-55.
// ===========================================================================
struct Operator {
    virtual ~Operator() = default;
    virtual int order() const = 0;
};

template <typename T>
struct AdjointOperator {
    virtual ~AdjointOperator() = default;
    virtual int order() const = 0;
    virtual void apply(const T* x, T* y, int t) = 0;          // Y := A X
    virtual void apply_adjoint(const T* x, T* y, int t) = 0;  // Y := A^H X
};

void panel_apply(int n, int t, const double* a, int lda, const double* x, int ldx, double* y, int ldy) {
    for (int c = 0; c < t; c++) {
        const double* src = x + (size_t)c * ldx;
        double* dst = y + (size_t)c * ldy;
        std::memset(dst, 0, sizeof(double) * (size_t)n);
        for (int j = 0; j < n; j++) {
            double s = src[j];
            if (s != 0.0) col_axpy(n, s, a + (size_t)j * lda, dst);
        }
    }
}
void panel_apply_transpose(int n, int t, const double* a, int lda, const double* x, int ldx, double* y,
                           int ldy) {
    for (int c = 0; c < t; c++) {
        const double* src = x + (size_t)c * ldx;
        double* dst = y + (size_t)c * ldy;
        for (int j = 0; j < n; j++) dst[j] = col_dot(n, a + (size_t)j * lda, src);
    }
}

struct DenseRealOperator : AdjointOperator<double> {
    int n, lda, power;
    const double* a;
    DenseRealOperator(int n_, const double* a_, int lda_, int p) : n(n_), lda(lda_), power(p), a(a_) {}
    int order() const override { return n; }
    void repeat(const double* x, double* y, int t, bool tr) {
        (tr ? panel_apply_transpose : panel_apply)(n, t, a, lda, x, n, y, n);
        if (power == 1) return;
        std::vector<double> staging((size_t)n * t);
        for (int step = 1; step < power; step++) {
            std::memcpy(staging.data(), y, sizeof(double) * (size_t)n * t);
            (tr ? panel_apply_transpose : panel_apply)(n, t, a, lda, staging.data(), n, y, n);
        }
    }
    void apply(const double* x, double* y, int t) override { repeat(x, y, t, false); }
    void apply_adjoint(const double* x, double* y, int t) override { repeat(x, y, t, true); }
};

struct DenseComplexOperator : AdjointOperator<cplx> {
    int n, power;
    std::vector<double> re, im;
    DenseComplexOperator(int n_, const cplx* a, int lda, int p) : n(n_), power(p) {
        re.resize((size_t)n * n);
        im.resize((size_t)n * n);
        split(n, n, a, lda, re.data(), im.data());
    }
    int order() const override { return n; }
    void repeat(const cplx* x, cplx* y, int t, bool adj) {
        if (n == 0 || t == 0) return;
        std::vector<double> st((size_t)n * 2 * t), p((size_t)n * 2 * t), q((size_t)n * 2 * t);
        auto split_into = [&](const cplx* src) {
            for (int j = 0; j < t; j++)
                for (int i = 0; i < n; i++) {
                    st[(size_t)j * n + i] = src[(size_t)j * n + i].re;
                    st[(size_t)(t + j) * n + i] = src[(size_t)j * n + i].im;
                }
        };
        split_into(x);
        for (int step = 0; step < power; step++) {
            if (step > 0) split_into(y);
            (adj ? panel_apply_transpose : panel_apply)(n, 2 * t, re.data(), n, st.data(), n, p.data(), n);
            (adj ? panel_apply_transpose : panel_apply)(n, 2 * t, im.data(), n, st.data(), n, q.data(), n);
            for (int j = 0; j < t; j++)
                for (int i = 0; i < n; i++) {
                    double pr = p[(size_t)j * n + i], pi = p[(size_t)(t + j) * n + i];
                    double qr = q[(size_t)j * n + i], qi = q[(size_t)(t + j) * n + i];
                    y[(size_t)j * n + i] = adj ? cplx{pr + qi, pi - qr} : cplx{pr - qi, pi + qr};
                }
        }
    }
    void apply(const cplx* x, cplx* y, int t) override { repeat(x, y, t, false); }
    void apply_adjoint(const cplx* x, cplx* y, int t) override { repeat(x, y, t, true); }
};

struct LuInverseRealOperator : AdjointOperator<double> {
    int n, lda;
    const double* lu;
    const int* piv;
    LuInverseRealOperator(int n_, const double* lu_, int lda_, const int* p) : n(n_), lda(lda_), lu(lu_), piv(p) {}
    int order() const override { return n; }
    // src/Tensile.Kernels/Lu.cs:336-378
    void apply(const double* x, double* y, int t) override {
        std::memcpy(y, x, sizeof(double) * (size_t)n * t);
        swap_rows(y, n, 0, t, piv, 0, n);
        solve_lower_unit(n, t, lu, lda, y, n);
        solve_upper(n, t, lu, lda, y, n);
    }
    void apply_adjoint(const double* x, double* y, int t) override {
        std::memcpy(y, x, sizeof(double) * (size_t)n * t);
        solve_upper_transposed(n, t, lu, lda, y, n);
        solve_lower_unit_transposed(n, t, lu, lda, y, n);
        unswap_rows(y, n, 0, t, piv, 0, n);
    }
};

struct LuInverseComplexOperator : AdjointOperator<cplx> {
    int n, lda;
    const cplx* lu;
    const int* piv;
    LuInverseComplexOperator(int n_, const cplx* lu_, int lda_, const int* p) : n(n_), lda(lda_), lu(lu_), piv(p) {}
    int order() const override { return n; }
    // src/Tensile/BlockedLu.cs:105-141
    void apply(const cplx* x, cplx* y, int t) override {
        std::memcpy(y, x, sizeof(cplx) * (size_t)n * t);
        swap_rows(y, n, 0, t, piv, 0, n);
        zsolve_lower_unit(n, t, lu, lda, y, n);
        zsolve_upper(n, t, lu, lda, y, n);
    }
    void apply_adjoint(const cplx* x, cplx* y, int t) override {
        std::memcpy(y, x, sizeof(cplx) * (size_t)n * t);
        zsolve_upper_adjoint(n, t, lu, lda, y, n);
        zsolve_lower_unit_adjoint(n, t, lu, lda, y, n);
        unswap_rows(y, n, 0, t, piv, 0, n);
    }
};

// ===========================================================================
// Block 1-norm estimator. src/Tensile/NormEstimate.cs:104-411.
// ===========================================================================
template <typename T>
bool is_parallel(const T* u, const T* v, int n) {
    bool same = true, opposite = true;
    for (int i = 0; i < n; i++) {
        if (!(u[i] == v[i])) same = false;
        if (!(u[i] == -v[i])) opposite = false;
        if (!same && !opposite) return false;
    }
    return true;
}

template <typename T>
bool is_parallel_to_any(int n, const T* column, const T* panel, int count) {
    for (int j = 0; j < count; j++)
        if (is_parallel<T>(column, panel + (size_t)j * n, n)) return true;
    return false;
}

template <typename K>
orc_normest_result normest(AdjointOperator<typename K::T>& op, int columns, int max_iterations, int seed) {
    using T = typename K::T;
    int n = op.order();
    if (n == 0) return {0.0, 0, 0};
    int t = std::clamp(columns, 1, n);
    int itmax = std::max(max_iterations, 2);
    size_t extent = (size_t)n * t;
    std::vector<T> x(extent), y(extent), s(extent), s_old(extent), z(extent);
    std::vector<double> h(n), keys(n);
    std::vector<int> order(n), scratch(n), current(t);
    std::vector<char> used(n, 0);
    NetRandom rng(seed);

    auto fill_signs = [&](T* panel, int start) {
        for (int i = 0; i < n; i++) panel[start + i] = rng.next(2) == 0 ? K::neg(K::one()) : K::one();
    };
    // InitialProbe, :281-299
    for (int i = 0; i < n; i++) x[i] = K::one();
    for (int j = 1; j < t; j++)
        for (int attempt = 0; attempt < 8; attempt++) {
            fill_signs(x.data(), j * n);
            if (!is_parallel_to_any<T>(n, x.data() + (size_t)j * n, x.data(), j)) break;
        }
    {
        double sc = 1.0 / n;
        T scale = K::scale(K::one(), sc);  // CreateTruncating(1.0/n)
        for (size_t i = 0; i < extent; i++) x[i] = K::mul(x[i], scale);
    }

    auto column_one_norm = [&](const T* p) {
        double sum = 0.0;
        for (int i = 0; i < n; i++) sum += K::magnitude(p[i]);
        return sum;
    };

    double est = 0.0, est_old = 0.0;
    int best_index = -1, iterations = 0, products = 0;
    for (int k = 1;; k++) {
        iterations = k;
        op.apply(x.data(), y.data(), t);
        products += t;
        int argmax = 0;
        est = column_one_norm(y.data());
        for (int j = 1; j < t; j++) {
            double v = column_one_norm(y.data() + (size_t)j * n);
            if (v > est) {
                est = v;
                argmax = j;
            }
        }
        if (k >= 2 && (est > est_old || k == 2)) best_index = current[argmax];
        if (k >= 2 && est <= est_old) {
            est = est_old;
            break;
        }
        est_old = est;
        if (k > itmax) break;
        std::swap(s, s_old);
        for (size_t i = 0; i < extent; i++) s[i] = K::sign(y[i]);
        if (K::discrete && t > 1) {
            bool all_parallel = true;
            for (int j = 0; j < t; j++)
                if (!is_parallel_to_any<T>(n, s.data() + (size_t)j * n, s_old.data(), t)) {
                    all_parallel = false;
                    break;
                }
            if (all_parallel) break;
            // MakeColumnsDistinct, :357-370
            for (int j = 0; j < t; j++)
                for (int attempt = 0; attempt < 8; attempt++) {
                    if (!is_parallel_to_any<T>(n, s.data() + (size_t)j * n, s.data(), j) &&
                        !is_parallel_to_any<T>(n, s.data() + (size_t)j * n, s_old.data(), t))
                        break;
                    fill_signs(s.data(), j * n);
                }
        }
        op.apply_adjoint(s.data(), z.data(), t);
        products += t;
        for (int i = 0; i < n; i++) {
            double best = 0.0;
            for (int j = 0; j < t; j++) best = net_max(best, K::magnitude(z[(size_t)j * n + i]));
            h[i] = best;
        }
        if (k >= 2 && best_index >= 0) {
            double largest = 0.0;
            for (int i = 0; i < n; i++) largest = net_max(largest, h[i]);
            if (largest == h[best_index]) break;
        }
        for (int i = 0; i < n; i++) {
            keys[i] = -h[i];
            order[i] = i;
        }
        NetSort{keys.data(), order.data()}.sort(n);
        if (t > 1) {
            bool all_used = true;
            for (int j = 0; j < t; j++)
                if (!used[order[j]]) {
                    all_used = false;
                    break;
                }
            if (all_used) break;
            int at = 0;
            for (int i = 0; i < n; i++)
                if (!used[order[i]]) scratch[at++] = order[i];
            for (int i = 0; i < n; i++)
                if (used[order[i]]) scratch[at++] = order[i];
            std::copy(scratch.begin(), scratch.end(), order.begin());
        }
        std::fill(x.begin(), x.end(), K::zero());
        for (int j = 0; j < t; j++) {
            int index = order[j];
            current[j] = index;
            used[index] = 1;
            x[(size_t)j * n + index] = K::one();
        }
    }
    return {est, iterations, products};
}

// ===========================================================================
// Matrix exponential. src/Tensile/MatrixExponential.cs:181-558.
// ===========================================================================
const double Theta3 = 1.495585217958292e-2;
const double Theta5 = 2.539398330063230e-1;
const double Theta7 = 9.504178996162932e-1;
const double Theta9 = 2.097847961257068e0;
const double ScalingThreshold = 4.25;
const double UnitRoundoff = 1.1102230246251565e-16;
const double Pade3[] = {120, 60, 12, 1};
const double Pade5[] = {30240, 15120, 3360, 420, 30, 1};
const double Pade7[] = {17297280, 8648640, 1995840, 277200, 25200, 1512, 56, 1};
const double Pade9[] = {17643225600.0, 8821612800.0, 2075673600.0, 302702400.0, 30270240.0,
                        2162160.0,     110880.0,     3960.0,       90.0,        1.0};
const double Pade13[] = {64764752532480000.0, 32382376266240000.0, 7771770303897600.0,
                         1187353796428800.0,  129060195264000.0,   10559470521600.0,
                         670442572800.0,      33522128640.0,       1323241920.0,
                         40840800.0,          960960.0,            16380.0,
                         182.0,               1.0};

double abs_coeff_reciprocal(int m) {
    switch (m) {
        case 3: return 100800.0;
        case 5: return 10059033600.0;
        case 7: return 4487938430976000.0;
        case 9: return 5914384781877411840000.0;
        default: return 113250775606021113483283660800000000.0;
    }
}

template <typename K>
struct Mat {
    using T = typename K::T;
    int n;
    std::vector<T> v;
    explicit Mat(int n_) : n(n_), v((size_t)n_ * n_, K::zero()) {}
    T* p() { return v.data(); }
    const T* p() const { return v.data(); }
    T& at(int i, int j) { return v[(size_t)j * n + i]; }
};

template <typename K>
Mat<K> product(const Mat<K>& x, const Mat<K>& y) {
    Mat<K> r(x.n);
    K::gemm(x.n, x.n, x.n, x.p(), x.n, y.p(), y.n, K::zero(), r.p(), r.n);
    return r;
}
template <typename K>
Mat<K> identity(int n, double scale) {
    Mat<K> r(n);
    for (int i = 0; i < n; i++) r.at(i, i) = K::scale(K::one(), scale);  // CreateTruncating(scale)
    return r;
}
template <typename K>
Mat<K> scaled(const Mat<K>& s, double f) {
    Mat<K> r(s.n);
    for (size_t i = 0; i < s.v.size(); i++) r.v[i] = K::scale(s.v[i], f);
    return r;
}
template <typename K>
void add_scaled(Mat<K>& t, const Mat<K>& s, double f) {
    for (size_t i = 0; i < s.v.size(); i++) t.v[i] = K::add(t.v[i], K::scale(s.v[i], f));
}

template <typename K>
double one_norm_abs_power(const Mat<K>& a, int p) {
    int n = a.n;
    std::vector<double> mag((size_t)n * n), row(n, 1.0), next(n);
    for (size_t i = 0; i < mag.size(); i++) mag[i] = K::magnitude(a.v[i]);
    for (int step = 0; step < p; step++) {
        for (int j = 0; j < n; j++) {
            const double* col = mag.data() + (size_t)j * n;
            double sum = 0.0;
            for (int i = 0; i < n; i++) sum += row[i] * col[i];
            next[j] = sum;
        }
        std::swap(row, next);
    }
    double best = 0.0;
    for (int j = 0; j < n; j++) best = net_max(best, row[j]);
    return best;
}

template <typename K>
int ell(const Mat<K>& a, int m) {
    double a_norm = K::one_norm(a.n, a.n, a.p(), a.n);
    if (a_norm == 0.0) return 0;
    double apn = one_norm_abs_power(a, 2 * m + 1);
    if (apn == 0.0) return 0;
    double alpha = apn / (a_norm * abs_coeff_reciprocal(m));
    int value = (int)std::ceil(std::log2(alpha / UnitRoundoff) / (2 * m));
    return std::max(value, 0);
}

template <typename K>
struct PowerOp;
template <>
struct PowerOp<RealK> {
    static double est(const Mat<RealK>& a, int p, int t = 2) {
        DenseRealOperator op(a.n, a.p(), a.n, p);
        return normest<RealK>(op, t, 5, 20260915).value;
    }
};
template <>
struct PowerOp<ComplexK> {
    static double est(const Mat<ComplexK>& a, int p, int t = 2) {
        DenseComplexOperator op(a.n, a.p(), a.n, p);
        return normest<ComplexK>(op, t, 5, 20260915).value;
    }
};

template <typename K>
struct LuOf;
template <>
struct LuOf<RealK> {
    static void factor(Mat<RealK>& a, std::vector<int>& piv, orc_lu_info* info) {
        dgetrf_impl(a.n, a.n, a.p(), a.n, 0, piv.data(), info);
    }
    static void solve(const Mat<RealK>& lu, const std::vector<int>& piv, Mat<RealK>& b) {
        swap_rows(b.p(), b.n, 0, b.n, piv.data(), 0, b.n);
        solve_lower_unit(b.n, b.n, lu.p(), lu.n, b.p(), b.n);
        solve_upper(b.n, b.n, lu.p(), lu.n, b.p(), b.n);
    }
};
template <>
struct LuOf<ComplexK> {
    static void factor(Mat<ComplexK>& a, std::vector<int>& piv, orc_lu_info* info) {
        zgetrf_impl(a.n, a.n, a.p(), a.n, 0, piv.data(), info);
    }
    static void solve(const Mat<ComplexK>& lu, const std::vector<int>& piv, Mat<ComplexK>& b) {
        swap_rows(b.p(), b.n, 0, b.n, piv.data(), 0, b.n);
        zsolve_lower_unit(b.n, b.n, lu.p(), lu.n, b.p(), b.n);
        zsolve_upper(b.n, b.n, lu.p(), lu.n, b.p(), b.n);
    }
};

// SolvePade, :372-405: (V - U) X = (V + U). False when the denominator is singular.
template <typename K>
bool solve_pade_exact(const Mat<K>& u, const Mat<K>& v, Mat<K>& out);

template <>
bool solve_pade_exact<RealK>(const Mat<RealK>& u, const Mat<RealK>& v, Mat<RealK>& out) {
    int n = u.n;
    Mat<RealK> den(n), num(n);
    for (size_t i = 0; i < u.v.size(); i++) {
        den.v[i] = v.v[i] - u.v[i];
        num.v[i] = v.v[i] + u.v[i];
    }
    std::vector<int> piv(n);
    orc_lu_info info;
    LuOf<RealK>::factor(den, piv, &info);
    if (info.singular_column >= 0) return false;
    LuOf<RealK>::solve(den, piv, num);
    out = std::move(num);
    return true;
}
template <>
bool solve_pade_exact<ComplexK>(const Mat<ComplexK>& u, const Mat<ComplexK>& v, Mat<ComplexK>& out) {
    int n = u.n;
    Mat<ComplexK> den(n), num(n);
    for (size_t i = 0; i < u.v.size(); i++) {
        den.v[i] = csub(v.v[i], u.v[i]);
        num.v[i] = cadd(v.v[i], u.v[i]);
    }
    std::vector<int> piv(n);
    orc_lu_info info;
    LuOf<ComplexK>::factor(den, piv, &info);
    if (info.singular_column >= 0) return false;
    LuOf<ComplexK>::solve(den, piv, num);
    out = std::move(num);
    return true;
}

// EvaluateLowDegree, :284-315
template <typename K>
bool evaluate_low(const double* b, int m, const Mat<K>& a, const Mat<K>& a2, const Mat<K>& a4,
                  const Mat<K>& a6, const Mat<K>* a8, Mat<K>& out) {
    int n = a.n;
    Mat<K> w = identity<K>(n, b[1]);
    add_scaled(w, a2, b[3]);
    if (m >= 5) add_scaled(w, a4, b[5]);
    if (m >= 7) add_scaled(w, a6, b[7]);
    if (m >= 9) add_scaled(w, *a8, b[9]);
    Mat<K> u = product(a, w);
    Mat<K> v = identity<K>(n, b[0]);
    add_scaled(v, a2, b[2]);
    if (m >= 5) add_scaled(v, a4, b[4]);
    if (m >= 7) add_scaled(v, a6, b[6]);
    if (m >= 9) add_scaled(v, *a8, b[8]);
    return solve_pade_exact<K>(u, v, out);
}

// EvaluateDegree13, :323-360
template <typename K>
bool evaluate13(const Mat<K>& a, const Mat<K>& a2, const Mat<K>& a4, const Mat<K>& a6, Mat<K>& out) {
    const double* b = Pade13;
    int n = a.n;
    Mat<K> inner = scaled(a6, b[13]);
    add_scaled(inner, a4, b[11]);
    add_scaled(inner, a2, b[9]);
    Mat<K> w = identity<K>(n, b[1]);
    add_scaled(w, a2, b[3]);
    add_scaled(w, a4, b[5]);
    add_scaled(w, a6, b[7]);
    K::gemm(n, n, n, a6.p(), n, inner.p(), n, K::one(), w.p(), n);
    Mat<K> u = product(a, w);
    Mat<K> inner_even = scaled(a6, b[12]);
    add_scaled(inner_even, a4, b[10]);
    add_scaled(inner_even, a2, b[8]);
    Mat<K> v = identity<K>(n, b[0]);
    add_scaled(v, a2, b[2]);
    add_scaled(v, a4, b[4]);
    add_scaled(v, a6, b[6]);
    K::gemm(n, n, n, a6.p(), n, inner_even.p(), n, K::one(), v.p(), n);
    return solve_pade_exact<K>(u, v, out);
}

template <typename K>
int scaling_and_squaring(const Mat<K>& a, Mat<K>& out, orc_expm_info* info) {
    int n = a.n;
    Mat<K> a2 = product(a, a);
    Mat<K> a4 = product(a2, a2);
    Mat<K> a6 = product(a2, a4);
    double d4 = std::pow(K::one_norm(n, n, a4.p(), n), 1.0 / 4.0);
    double d6 = std::pow(K::one_norm(n, n, a6.p(), n), 1.0 / 6.0);
    double eta1 = net_max(d4, d6);
    info->d4 = d4;
    info->d6 = d6;
    info->eta1 = eta1;
    info->squarings = 0;
    if (eta1 < Theta3 && ell(a, 3) == 0) {
        info->degree = 3;
        return evaluate_low<K>(Pade3, 3, a, a2, a4, a6, nullptr, out) ? 0 : 2;
    }
    if (eta1 < Theta5 && ell(a, 5) == 0) {
        info->degree = 5;
        return evaluate_low<K>(Pade5, 5, a, a2, a4, a6, nullptr, out) ? 0 : 2;
    }
    double d8 = std::pow(PowerOp<K>::est(a, 8), 1.0 / 8.0);
    double eta3 = net_max(d6, d8);
    info->d8 = d8;
    info->eta3 = eta3;
    if (eta3 < Theta7 && ell(a, 7) == 0) {
        info->degree = 7;
        return evaluate_low<K>(Pade7, 7, a, a2, a4, a6, nullptr, out) ? 0 : 2;
    }
    if (eta3 < Theta9 && ell(a, 9) == 0) {
        info->degree = 9;
        Mat<K> a8 = product(a4, a4);
        return evaluate_low<K>(Pade9, 9, a, a2, a4, a6, &a8, out) ? 0 : 2;
    }
    double d10 = std::pow(PowerOp<K>::est(a, 10), 1.0 / 10.0);
    double eta4 = net_max(d8, d10);
    double eta5 = net_min(eta3, eta4);
    info->d10 = d10;
    info->eta5 = eta5;
    int s = eta5 == 0.0 ? 0 : std::max((int)std::ceil(std::log2(eta5 / ScalingThreshold)), 0);
    Mat<K> sc = scaled(a, std::ldexp(1.0, -s));
    s += ell(sc, 13);
    double factor = std::ldexp(1.0, -s);
    Mat<K> b = scaled(a, factor);
    Mat<K> b2 = scaled(a2, factor * factor);
    Mat<K> b4 = scaled(a4, std::pow(factor, 4));
    Mat<K> b6 = scaled(a6, std::pow(factor, 6));
    info->degree = 13;
    info->squarings = s;
    Mat<K> x(n);
    if (!evaluate13<K>(b, b2, b4, b6, x)) return 2;
    Mat<K> sq(n);
    for (int i = 0; i < s; i++) {
        K::gemm(n, n, n, x.p(), n, x.p(), n, K::zero(), sq.p(), n);
        std::swap(x, sq);
    }
    out = std::move(x);
    return 0;
}

template <typename K>
int expm(int n, const typename K::T* a, int lda, typename K::T* out, int ldo, orc_expm_info* info) {
    orc_expm_info local{};
    if (!info) info = &local;
    *info = orc_expm_info{};
    if (n < 0) return 1;
    if (n <= 1) {
        if (n == 1) out[0] = K::exp(a[0]);
        return 0;
    }
    Mat<K> am(n);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) am.at(i, j) = a[(size_t)j * lda + i];
    Mat<K> r(n);
    int rc = scaling_and_squaring<K>(am, r, info);
    if (rc != 0) return rc;
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) out[(size_t)j * ldo + i] = r.at(i, j);
    return 0;
}

// ===========================================================================
// Exponential action. src/Tensile/MatrixExponentialAction.cs:149-485,
// src/Tensile/MatrixExponentialAction.Complex.cs:34-126.
// ===========================================================================
const int Degrees[] = {1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18,
                       19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 35, 40, 45, 50, 55};
const double Thetas[] = {2.29e-16, 2.58e-8, 1.39e-5, 3.40e-4, 2.40e-3, 9.07e-3, 2.38e-2,
                         5.00e-2,  8.96e-2, 1.44e-1, 2.14e-1, 3.00e-1, 4.00e-1, 5.14e-1,
                         6.41e-1,  7.81e-1, 9.31e-1, 1.09,    1.26,    1.44,    1.62,
                         1.82,     2.01,    2.22,    2.43,    2.64,    2.86,    3.08,
                         3.31,     3.54,    4.7,     6.0,     7.2,     8.5,     9.9};
constexpr int NDegrees = 35, MaxDegree = 55, MaxPower = 8, EllProbe = 2;

// SelectParameters, :347-398. Returns 8 when the cost is not countable.
template <typename AlphaFn>
int select_parameters(double scaled_norm, bool have_alpha, AlphaFn alpha, double scale, int columns,
                      int* m_out, int* s_out) {
    int best_degree = 0;
    double best_scaling = 0.0, best_cost = std::numeric_limits<double>::infinity();
    auto consider = [&](int index, double norm) {
        double scaling = std::ceil(norm / Thetas[index]);
        double cost = Degrees[index] * scaling;
        if (cost >= best_cost) return;
        best_cost = cost;
        best_degree = Degrees[index];
        best_scaling = scaling;
    };
    double a = 2.0 * EllProbe * MaxPower * (MaxPower + 3);
    double b = Thetas[NDegrees - 1] / (columns * (double)MaxDegree);
    bool cond313 = scaled_norm <= a * b;
    if (!have_alpha || cond313) {
        for (int index = 0; index < NDegrees; index++) consider(index, scaled_norm);
    } else {
        for (int p = 2; p <= MaxPower; p++) {
            double alpha_p = scale * alpha(p);
            for (int index = 0; index < NDegrees; index++) {
                if (Degrees[index] < (p * (p - 1)) - 1) continue;
                consider(index, alpha_p);
            }
        }
    }
    double steps = std::max(best_scaling, 1.0);
    if (!std::isfinite(best_cost) || steps > 2147483647.0) return 8;
    *m_out = best_degree;
    *s_out = (int)steps;
    return 0;
}

template <typename K>
int expmv_dense(int n, const typename K::T* a, int lda, int ncols, const typename K::T* b, int ldb,
                double t, typename K::T* out, int ldo, orc_expmv_info* info) {
    using T = typename K::T;
    orc_expmv_info local{};
    if (!info) info = &local;
    *info = orc_expmv_info{};
    if (n == 0 || ncols == 0) {
        if (b)
            for (int j = 0; j < ncols; j++)
                for (int i = 0; i < n; i++) out[(size_t)j * ldo + i] = b[(size_t)j * ldb + i];
        return 0;
    }
    // Trace shift (:138-139; complex :57-60).
    Mat<K> sh(n);
    T trace = K::zero();
    for (int i = 0; i < n; i++) trace = K::add(trace, a[(size_t)i * lda + i]);
    T mu;
    if constexpr (std::is_same_v<T, double>)
        mu = trace / n;
    else
        mu = cplx{trace.re / n, trace.im / n};
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) sh.at(i, j) = a[(size_t)j * lda + i];
    for (int i = 0; i < n; i++) sh.at(i, i) = K::add(sh.at(i, i), K::neg(mu));

    double one_norm = K::one_norm(n, n, sh.p(), n);
    double d[MaxPower + 2];
    for (double& v : d) v = std::numeric_limits<double>::quiet_NaN();
    auto D = [&](int p) {
        if (std::isnan(d[p])) d[p] = std::pow(PowerOp<K>::est(sh, p, EllProbe), 1.0 / p);
        return d[p];
    };
    auto alpha = [&](int p) { return net_max(D(p), D(p + 1)); };

    double scale = std::fabs(t);
    double scaled_norm = scale * one_norm;
    int m, s;
    if (scaled_norm == 0.0) {
        m = 0;
        s = 1;
    } else {
        int rc = select_parameters(scaled_norm, true, alpha, scale, ncols, &m, &s);
        if (rc) return rc;
    }
    info->degree = m;
    info->scaling = s;
    if (!b) return 0;  // the parameters only (orc_{d,z}expmv_params)

    size_t ext = (size_t)n * ncols;
    std::vector<T> f(ext), work(ext), next(ext);
    for (int j = 0; j < ncols; j++)
        for (int i = 0; i < n; i++) f[(size_t)j * n + i] = work[(size_t)j * n + i] = b[(size_t)j * ldb + i];
    T eta = K::exp(K::div_real(K::scale(mu, t), (double)s));
    typename std::conditional<std::is_same_v<T, double>, DenseRealOperator, DenseComplexOperator>::type op(
        n, sh.p(), n, 1);
    for (int i = 0; i < s; i++) {
        double c1 = K::inf_norm(n, ncols, work.data(), n);
        for (int j = 0; j < m; j++) {
            double coefficient = t / (s * (double)(j + 1));
            op.apply(work.data(), next.data(), ncols);
            for (size_t q = 0; q < ext; q++) work[q] = K::scale(next[q], coefficient);
            double c2 = K::inf_norm(n, ncols, work.data(), n);
            for (size_t q = 0; q < ext; q++) f[q] = K::add(f[q], work[q]);
            info->applications++;
            if (c1 + c2 <= UnitRoundoff * K::inf_norm(n, ncols, f.data(), n)) {
                info->early_exits++;
                break;
            }
            c1 = c2;
        }
        if (!K::eq(eta, K::one()))
            for (size_t q = 0; q < ext; q++) f[q] = K::mul(f[q], eta);
        work = f;
    }
    for (int j = 0; j < ncols; j++)
        for (int i = 0; i < n; i++) out[(size_t)j * ldo + i] = f[(size_t)j * n + i];
    return 0;
}

// The matrix-free Expmv (MatrixExponentialAction.Expmv(ILinearOperator<T>, B, t,
// oneNormBound), src/Tensile/MatrixExponentialAction.cs:203-230 and
// .Complex.cs:85-111): no trace, so mu = 0; the caller's bound on ||A||_1; no
// estimator, so the crude bound over every degree (alpha null in
// SelectParameters, :347-398); then Run (:239-320) with op.Apply. The
// operator here is a dense A applied as DenseMatrixOperator does.
template <typename K>
int expmv_matrix_free(int n, const typename K::T* a, int lda, int ncols, const typename K::T* b, int ldb, double t,
                      double bound, typename K::T* out, int ldo, orc_expmv_info* info) {
    using T = typename K::T;
    orc_expmv_info local{};
    if (!info) info = &local;
    *info = orc_expmv_info{};
    if (n == 0 || ncols == 0) {
        for (int j = 0; j < ncols; j++)
            for (int i = 0; i < n; i++) out[(size_t)j * ldo + i] = b[(size_t)j * ldb + i];
        return 0;
    }
    Mat<K> am(n);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) am.at(i, j) = a[(size_t)j * lda + i];
    double scale = std::fabs(t);
    double scaled_norm = scale * bound;
    int m, s;
    if (scaled_norm == 0.0) {
        m = 0;
        s = 1;
    } else {
        auto no_alpha = [](int) { return 0.0; };
        int rc = select_parameters(scaled_norm, false, no_alpha, scale, ncols, &m, &s);
        if (rc) return rc;
    }
    info->degree = m;
    info->scaling = s;
    size_t ext = (size_t)n * ncols;
    std::vector<T> f(ext), work(ext), next(ext);
    for (int j = 0; j < ncols; j++)
        for (int i = 0; i < n; i++) f[(size_t)j * n + i] = work[(size_t)j * n + i] = b[(size_t)j * ldb + i];
    typename std::conditional<std::is_same_v<T, double>, DenseRealOperator, DenseComplexOperator>::type op(
        n, am.p(), n, 1);
    for (int i = 0; i < s; i++) {
        double c1 = K::inf_norm(n, ncols, work.data(), n);
        for (int j = 0; j < m; j++) {
            double coefficient = t / (s * (double)(j + 1));
            op.apply(work.data(), next.data(), ncols);
            for (size_t q = 0; q < ext; q++) work[q] = K::scale(next[q], coefficient);
            double c2 = K::inf_norm(n, ncols, work.data(), n);
            for (size_t q = 0; q < ext; q++) f[q] = K::add(f[q], work[q]);
            info->applications++;
            if (c1 + c2 <= UnitRoundoff * K::inf_norm(n, ncols, f.data(), n)) {
                info->early_exits++;
                break;
            }
            c1 = c2;
        }
        work = f;  // eta = exp(0) = 1: no scaling
    }
    for (int j = 0; j < ncols; j++)
        for (int i = 0; i < n; i++) out[(size_t)j * ldo + i] = f[(size_t)j * n + i];
    return 0;
}

}  // namespace

// ===========================================================================
// C API
// ===========================================================================
extern "C" {

struct orc_random {
    NetRandom r;
};
orc_random* orc_random_new(int seed) { return new orc_random{NetRandom(seed)}; }
void orc_random_free(orc_random* r) { delete r; }
int orc_random_next(orc_random* r, int max_value) { return r->r.next(max_value); }
double orc_random_next_double(orc_random* r) { return r->r.sample(); }
void orc_sort_keys_items(int n, double* keys, int* items) { NetSort{keys, items}.sort(n); }

void orc_set_threads(int threads) { g_threads = threads; }
int orc_get_threads(void) { return threads_now(); }

int orc_dgemm(int m, int n, int k, double alpha, const double* a, int lda, const double* b, int ldb,
              double beta, double* c, int ldc, int multithreaded) {
    if (m < 0 || n < 0 || k < 0) return 1;
    dgemm_impl(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, multithreaded != 0);
    return 0;
}
int orc_zgemm(int m, int n, int k, const double* alpha, const double* a, int lda, const double* b,
              int ldb, const double* beta, double* c, int ldc, int multithreaded) {
    if (m < 0 || n < 0 || k < 0) return 1;
    if (m == 0 || n == 0) return 0;
    zgemm_impl(m, n, k, cplx{alpha[0], alpha[1]}, (const cplx*)a, lda, (const cplx*)b, ldb,
               cplx{beta[0], beta[1]}, (cplx*)c, ldc, multithreaded != 0);
    return 0;
}

double orc_dnorm1(int m, int n, const double* a, int lda) { return one_norm_real(m, n, a, lda); }
double orc_dnorminf(int m, int n, const double* a, int lda) { return inf_norm_real(m, n, a, lda); }
double orc_dnormfro(int m, int n, const double* a, int lda) {
    double total = 0.0;
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) {
            double v = a[(size_t)j * lda + i];
            total += v * v;
        }
    return std::sqrt(total);
}
double orc_znorm1(int m, int n, const double* a, int lda) { return one_norm_complex(m, n, (const cplx*)a, lda); }
double orc_znorminf(int m, int n, const double* a, int lda) { return inf_norm_complex(m, n, (const cplx*)a, lda); }
double orc_zabs(double re, double im) { return cabs_net(cplx{re, im}); }

int orc_dgetrf(int m, int n, double* a, int lda, int nb, int* pivots, orc_lu_info* info) {
    if (m < 0 || n < 0) return 1;
    dgetrf_impl(m, n, a, lda, nb, pivots, info);
    return 0;
}
int orc_zgetrf(int m, int n, double* a, int lda, int nb, int* pivots, orc_lu_info* info) {
    if (m < 0 || n < 0) return 1;
    zgetrf_impl(m, n, (cplx*)a, lda, nb, pivots, info);
    return 0;
}
// KernelEntry.SolveUpper .. SolveLowerUnitTransposed (src/Tensile.Kernels/KernelEntry.cs:98-173).
int orc_dtrsolve(int kind, int m, int n, const double* a, int lda, double* b, int ldb) {
    if (m == 0 || n == 0) return 0;
    switch (kind) {
        case 0: solve_upper(m, n, a, lda, b, ldb); return 0;
        case 1: solve_upper_transposed(m, n, a, lda, b, ldb); return 0;
        case 2: solve_lower(m, n, a, lda, b, ldb); return 0;
        case 3: solve_lower_transposed(m, n, a, lda, b, ldb); return 0;
        case 4: solve_lower_unit(m, n, a, lda, b, ldb); return 0;
        case 5: solve_lower_unit_transposed(m, n, a, lda, b, ldb); return 0;
        default: return 1;
    }
}

// BlockedLu's generic solves over Complex (src/Tensile/BlockedLu.cs:283-373).
int orc_ztrsolve(int kind, int m, int n, const double* a, int lda, double* b, int ldb) {
    if (m == 0 || n == 0) return 0;
    const cplx* A = reinterpret_cast<const cplx*>(a);
    cplx* B = reinterpret_cast<cplx*>(b);
    switch (kind) {
        case 0: zsolve_upper(m, n, A, lda, B, ldb); return 0;
        case 1: zsolve_upper_adjoint(m, n, A, lda, B, ldb); return 0;
        case 4: zsolve_lower_unit(m, n, A, lda, B, ldb); return 0;
        case 5: zsolve_lower_unit_adjoint(m, n, A, lda, B, ldb); return 0;
        default: return 1;
    }
}

// KernelEntry.MultiplyPanel / MultiplyPanelTransposed (KernelEntry.cs:176-201,
// PanelProduct.cs:25-55).
int orc_dpanel(int transposed, int n, int t, const double* a, int lda, const double* x, int ldx, double* y, int ldy) {
    if (n == 0 || t == 0) return 0;
    (transposed ? panel_apply_transpose : panel_apply)(n, t, a, lda, x, ldx, y, ldy);
    return 0;
}

// ComplexDenseOperator.Apply / ApplyAdjoint at power 1 (src/Tensile/LinearOperators.cs:194-293).
int orc_zpanel(int adjoint, int n, int t, const double* a, int lda, const double* x, int ldx, double* y, int ldy) {
    if (n == 0 || t == 0) return 0;
    DenseComplexOperator op(n, reinterpret_cast<const cplx*>(a), lda, 1);
    std::vector<cplx> xs((size_t)n * t), ys((size_t)n * t);
    for (int j = 0; j < t; j++)
        for (int i = 0; i < n; i++) xs[(size_t)j * n + i] = reinterpret_cast<const cplx*>(x)[(size_t)j * ldx + i];
    if (adjoint) op.apply_adjoint(xs.data(), ys.data(), t);
    else op.apply(xs.data(), ys.data(), t);
    for (int j = 0; j < t; j++)
        for (int i = 0; i < n; i++) reinterpret_cast<cplx*>(y)[(size_t)j * ldy + i] = ys[(size_t)j * n + i];
    return 0;
}

int orc_dgetrs(int n, int nrhs, const double* lu, int lda, const int* pivots, int singular_column,
               double* b, int ldb, int adjoint) {
    if (singular_column >= 0) return 2;
    if (n == 0 || nrhs == 0) return 0;
    if (!adjoint) {
        swap_rows(b, ldb, 0, nrhs, pivots, 0, n);
        solve_lower_unit(n, nrhs, lu, lda, b, ldb);
        solve_upper(n, nrhs, lu, lda, b, ldb);
    } else {
        solve_upper_transposed(n, nrhs, lu, lda, b, ldb);
        solve_lower_unit_transposed(n, nrhs, lu, lda, b, ldb);
        unswap_rows(b, ldb, 0, nrhs, pivots, 0, n);
    }
    return 0;
}
int orc_zgetrs(int n, int nrhs, const double* lu, int lda, const int* pivots, int singular_column,
               double* b, int ldb, int adjoint) {
    if (singular_column >= 0) return 2;
    if (n == 0 || nrhs == 0) return 0;
    const cplx* f = (const cplx*)lu;
    cplx* x = (cplx*)b;
    if (!adjoint) {
        swap_rows(x, ldb, 0, nrhs, pivots, 0, n);
        zsolve_lower_unit(n, nrhs, f, lda, x, ldb);
        zsolve_upper(n, nrhs, f, lda, x, ldb);
    } else {
        zsolve_upper_adjoint(n, nrhs, f, lda, x, ldb);
        zsolve_lower_unit_adjoint(n, nrhs, f, lda, x, ldb);
        unswap_rows(x, ldb, 0, nrhs, pivots, 0, n);
    }
    return 0;
}

int orc_dnormest_power(int n, const double* a, int lda, int power, int t, int itmax, int seed,
                       orc_normest_result* out) {
    if (n < 0 || power < 1) return 1;
    DenseRealOperator op(n, a, lda, power);
    *out = normest<RealK>(op, t, itmax, seed);
    return 0;
}
int orc_znormest_power(int n, const double* a, int lda, int power, int t, int itmax, int seed,
                       orc_normest_result* out) {
    if (n < 0 || power < 1) return 1;
    DenseComplexOperator op(n, (const cplx*)a, lda, power);
    *out = normest<ComplexK>(op, t, itmax, seed);
    return 0;
}
// src/Tensile/NormEstimate.cs:432-466
int orc_dgecon(int n, const double* lu, int lda, const int* pivots, int singular_column, double anorm,
               double* rcond) {
    if (singular_column >= 0 || anorm == 0.0 || n == 0) {
        *rcond = 0.0;
        return 0;
    }
    LuInverseRealOperator op(n, lu, lda, pivots);
    double inv = normest<RealK>(op, 2, 5, 20260915).value;
    *rcond = inv == 0.0 ? 0.0 : 1.0 / (anorm * inv);
    return 0;
}
int orc_zgecon(int n, const double* lu, int lda, const int* pivots, int singular_column, double anorm,
               double* rcond) {
    if (singular_column >= 0 || anorm == 0.0 || n == 0) {
        *rcond = 0.0;
        return 0;
    }
    LuInverseComplexOperator op(n, (const cplx*)lu, lda, pivots);
    double inv = normest<ComplexK>(op, 2, 5, 20260915).value;
    *rcond = inv == 0.0 ? 0.0 : 1.0 / (anorm * inv);
    return 0;
}

int orc_dexpm(int n, const double* a, int lda, double* out, int ldo, orc_expm_info* info) {
    return expm<RealK>(n, a, lda, out, ldo, info);
}
int orc_zexpm(int n, const double* a, int lda, double* out, int ldo, orc_expm_info* info) {
    return expm<ComplexK>(n, (const cplx*)a, lda, (cplx*)out, ldo, info);
}
int orc_dexpmv_bound(int n, const double* a, int lda, int ncols, const double* b, int ldb, double t, double bound,
                     double* out, int ldo, orc_expmv_info* info) {
    return expmv_matrix_free<RealK>(n, a, lda, ncols, b, ldb, t, bound, out, ldo, info);
}
int orc_zexpmv_bound(int n, const double* a, int lda, int ncols, const double* b, int ldb, double t, double bound,
                     double* out, int ldo, orc_expmv_info* info) {
    return expmv_matrix_free<ComplexK>(n, (const cplx*)a, lda, ncols, (const cplx*)b, ldb, t, bound, (cplx*)out, ldo,
                                       info);
}
int orc_dexpmv(int n, const double* a, int lda, int ncols, const double* b, int ldb, double t,
               double* out, int ldo, orc_expmv_info* info) {
    return expmv_dense<RealK>(n, a, lda, ncols, b, ldb, t, out, ldo, info);
}
int orc_zexpmv(int n, const double* a, int lda, int ncols, const double* b, int ldb, double t,
               double* out, int ldo, orc_expmv_info* info) {
    return expmv_dense<ComplexK>(n, (const cplx*)a, lda, ncols, (const cplx*)b, ldb, t, (cplx*)out, ldo,
                                 info);
}

// The (m, s) that Expmv selects for A, a panel of ncols columns and t,
// without running the recurrence.
int orc_dexpmv_params(int n, const double* a, int lda, int ncols, double t, orc_expmv_info* info) {
    return expmv_dense<RealK>(n, a, lda, ncols, nullptr, 0, t, nullptr, 0, info);
}
int orc_zexpmv_params(int n, const double* a, int lda, int ncols, double t, orc_expmv_info* info) {
    return expmv_dense<ComplexK>(n, (const cplx*)a, lda, ncols, nullptr, 0, t, nullptr, 0, info);
}

}  // extern "C"
