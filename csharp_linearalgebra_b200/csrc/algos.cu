// The reference's whole algorithms on the device: the Higham-Tisseur block
// 1-norm estimator, Al-Mohy & Higham 2009 scaling and squaring (Expm) and
// Al-Mohy & Higham 2011 truncated Taylor (Expmv).
//
// Control flow and every scalar decision run on the host in the reference's
// order, with the reference's constants; all O(n^2) and O(n^3) work runs in
// the sm_100a kernels. The estimator's bookkeeping (signs, column norms, the
// sort of candidates) is O(n t) and runs on the host over panels copied back
// from the device; the products run on the device.

#include "net_compat.h"
#include "tns_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

namespace tns {

namespace {

// ---------------------------------------------------------------------------
// Estimator element traits (IElementKernels<T> members the estimator uses,
// src/Tensile/ElementKernels.cs:137-157, src/Tensile/ComplexKernels.cs:111-129).
// ---------------------------------------------------------------------------
struct RealE {
    using T = double;
    static constexpr bool kDiscrete = true;
    static constexpr int kDoubles = 1;
    static T one() { return 1.0; }
    static T zero() { return 0.0; }
    static T neg(T x) { return -x; }
    static T mul(T a, T b) { return a * b; }
    static double magnitude(T x) { return std::fabs(x); }
    static T sign(T x) { return x >= 0.0 ? 1.0 : -1.0; }
    static bool eq(T a, T b) { return a == b; }
};
struct CplxE {
    using T = net::Cx;
    static constexpr bool kDiscrete = false;
    static constexpr int kDoubles = 2;
    static T one() { return {1.0, 0.0}; }
    static T zero() { return {0.0, 0.0}; }
    static T neg(T x) { return -x; }
    static T mul(T a, T b) { return net::mul(a, b); }
    static double magnitude(T x) { return net::abs(x); }
    static T sign(T x) {
        if (x == T{0.0, 0.0}) return {1.0, 0.0};
        double m = net::abs(x);
        return {x.re / m, x.im / m};
    }
    static bool eq(T a, T b) { return a == b; }
};

// An operator the estimator probes: applies A or A^H to an n x t panel held
// in host memory, through the device.
template <class TE>
struct Probe {
    virtual ~Probe() = default;
    virtual void apply(const typename TE::T* x, typename TE::T* y, int t, bool adjoint) = 0;
};

// Dense power operator (DenseMatrixOperator / ComplexDenseOperator,
// src/Tensile/LinearOperators.cs:89-293): p successive panel products.
template <class TE>
struct PowerProbe : Probe<TE> {
    Context& ctx;
    const DMat& a;
    int power;
    DBuf buf;
    PowerProbe(Context& c, const DMat& a_, int p, int t)
        : ctx(c), a(a_), power(p), buf(c, 2 * sizeof(double) * TE::kDoubles * (size_t)std::max(1, a_.rows) * t) {}
    void apply(const typename TE::T* x, typename TE::T* y, int t, bool adjoint) override {
        int n = a.rows;
        size_t bytes = sizeof(double) * TE::kDoubles * (size_t)n * t;
        double* d0 = buf.as<double>();
        double* d1 = d0 + (size_t)TE::kDoubles * n * t;
        TNS_CUDA(cudaMemcpyAsync(d0, x, bytes, cudaMemcpyHostToDevice, ctx.stream));
        for (int step = 0; step < power; ++step) {
            panel_product(ctx, a, d0, n, d1, n, t, adjoint);
            std::swap(d0, d1);
        }
        TNS_CUDA(cudaMemcpyAsync(y, d0, bytes, cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
    }
};

// Inverse of an LU factorization (LuInverseOperator,
// src/Tensile/LinearOperators.cs:303-350): apply = solve, adjoint = adjoint solve.
template <class TE>
struct LuInverseProbe : Probe<TE> {
    Context& ctx;
    const DMat& lu;
    const int* d_piv;
    DMat panel;
    LuInverseProbe(Context& c, const DMat& lu_, const int* piv, int t)
        : ctx(c), lu(lu_), d_piv(piv), panel(c, lu_.rows, t, lu_.cplx, "an estimator probe panel") {}
    void apply(const typename TE::T* x, typename TE::T* y, int t, bool adjoint) override {
        int n = lu.rows;
        size_t esz = sizeof(double) * TE::kDoubles;
        TNS_CUDA(cudaMemcpy2DAsync(panel.p, (size_t)panel.ld() * esz, x, (size_t)n * esz, (size_t)n * esz, t,
                                   cudaMemcpyHostToDevice, ctx.stream));
        getrs(ctx, lu, d_piv, panel, t, adjoint);
        TNS_CUDA(cudaMemcpy2DAsync(y, (size_t)n * esz, panel.p, (size_t)panel.ld() * esz, (size_t)n * esz, t,
                                   cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
    }
};

template <class TE>
bool is_parallel(const typename TE::T* u, const typename TE::T* v, int n) {
    bool same = true, opposite = true;
    for (int i = 0; i < n; ++i) {
        if (!TE::eq(u[i], v[i])) same = false;
        if (!TE::eq(u[i], TE::neg(v[i]))) opposite = false;
        if (!same && !opposite) return false;
    }
    return true;
}
template <class TE>
bool parallel_to_any(int n, const typename TE::T* col, const typename TE::T* panel, int count) {
    for (int j = 0; j < count; ++j)
        if (is_parallel<TE>(col, panel + (size_t)j * n, n)) return true;
    return false;
}

// NormEstimate.Estimate, src/Tensile/NormEstimate.cs:104-274.
template <class TE>
NormestResult estimate(Probe<TE>& op, int n, int columns, int max_iterations, int seed) {
    using T = typename TE::T;
    if (n == 0) return {};
    int t = std::clamp(columns, 1, n);
    int itmax = std::max(max_iterations, 2);
    size_t extent = (size_t)n * t;
    std::vector<T> x(extent), y(extent), s(extent), s_old(extent), z(extent);
    std::vector<double> h(n), keys(n);
    std::vector<int> order(n), scratch(n), current(t);
    std::vector<char> used(n, 0);
    net::Random rng(seed);
    auto fill_signs = [&](T* p) {
        for (int i = 0; i < n; ++i) p[i] = rng.next(2) == 0 ? TE::neg(TE::one()) : TE::one();
    };
    // InitialProbe, :281-299
    for (int i = 0; i < n; ++i) x[i] = TE::one();
    for (int j = 1; j < t; ++j)
        for (int attempt = 0; attempt < 8; ++attempt) {
            fill_signs(x.data() + (size_t)j * n);
            if (!parallel_to_any<TE>(n, x.data() + (size_t)j * n, x.data(), j)) break;
        }
    {
        T scale;
        if constexpr (TE::kDoubles == 1) scale = 1.0 / n;
        else scale = T{1.0 / n, 0.0};
        for (size_t i = 0; i < extent; ++i) x[i] = TE::mul(x[i], scale);
    }
    auto col_norm = [&](const T* p) {
        double sum = 0.0;
        for (int i = 0; i < n; ++i) sum += TE::magnitude(p[i]);
        return sum;
    };
    double est = 0.0, est_old = 0.0;
    int best_index = -1, iterations = 0, products = 0;
    for (int k = 1;; ++k) {
        iterations = k;
        op.apply(x.data(), y.data(), t, false);
        products += t;
        int argmax = 0;
        est = col_norm(y.data());
        for (int j = 1; j < t; ++j) {
            double v = col_norm(y.data() + (size_t)j * n);
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
        for (size_t i = 0; i < extent; ++i) s[i] = TE::sign(y[i]);
        if (TE::kDiscrete && t > 1) {
            bool all = true;
            for (int j = 0; j < t && all; ++j)
                if (!parallel_to_any<TE>(n, s.data() + (size_t)j * n, s_old.data(), t)) all = false;
            if (all) break;
            for (int j = 0; j < t; ++j)
                for (int attempt = 0; attempt < 8; ++attempt) {
                    if (!parallel_to_any<TE>(n, s.data() + (size_t)j * n, s.data(), j) &&
                        !parallel_to_any<TE>(n, s.data() + (size_t)j * n, s_old.data(), t))
                        break;
                    fill_signs(s.data() + (size_t)j * n);
                }
        }
        op.apply(s.data(), z.data(), t, true);
        products += t;
        for (int i = 0; i < n; ++i) {
            double best = 0.0;
            for (int j = 0; j < t; ++j) best = net::max(best, TE::magnitude(z[(size_t)j * n + i]));
            h[i] = best;
        }
        if (k >= 2 && best_index >= 0) {
            double largest = 0.0;
            for (int i = 0; i < n; ++i) largest = net::max(largest, h[i]);
            if (largest == h[best_index]) break;
        }
        for (int i = 0; i < n; ++i) {
            keys[i] = -h[i];
            order[i] = i;
        }
        net::sort_keys_items(n, keys.data(), order.data());
        if (t > 1) {
            bool all_used = true;
            for (int j = 0; j < t; ++j)
                if (!used[order[j]]) {
                    all_used = false;
                    break;
                }
            if (all_used) break;
            int at = 0;
            for (int i = 0; i < n; ++i)
                if (!used[order[i]]) scratch[at++] = order[i];
            for (int i = 0; i < n; ++i)
                if (used[order[i]]) scratch[at++] = order[i];
            std::copy(scratch.begin(), scratch.end(), order.begin());
        }
        std::fill(x.begin(), x.end(), TE::zero());
        for (int j = 0; j < t; ++j) {
            int index = order[j];
            current[j] = index;
            used[index] = 1;
            x[(size_t)j * n + index] = TE::one();
        }
    }
    return {est, iterations, products};
}

// ---------------------------------------------------------------------------
// Expm constants, src/Tensile/MatrixExponential.cs:50-110, 441-449.
// ---------------------------------------------------------------------------
const double kTheta3 = 1.495585217958292e-2;
const double kTheta5 = 2.539398330063230e-1;
const double kTheta7 = 9.504178996162932e-1;
const double kTheta9 = 2.097847961257068e0;
const double kScalingThreshold = 4.25;
const double kUnitRoundoff = 1.1102230246251565e-16;
const double kPade3[] = {120, 60, 12, 1};
const double kPade5[] = {30240, 15120, 3360, 420, 30, 1};
const double kPade7[] = {17297280, 8648640, 1995840, 277200, 25200, 1512, 56, 1};
const double kPade9[] = {17643225600.0, 8821612800.0, 2075673600.0, 302702400.0, 30270240.0,
                         2162160.0,     110880.0,     3960.0,       90.0,        1.0};
const double kPade13[] = {64764752532480000.0, 32382376266240000.0, 7771770303897600.0, 1187353796428800.0,
                          129060195264000.0,   10559470521600.0,    670442572800.0,     33522128640.0,
                          1323241920.0,        40840800.0,          960960.0,           16380.0,
                          182.0,               1.0};
const int kSeed = 20260915;

double abs_coeff_reciprocal(int m) {
    switch (m) {
        case 3: return 100800.0;
        case 5: return 10059033600.0;
        case 7: return 4487938430976000.0;
        case 9: return 5914384781877411840000.0;
        default: return 113250775606021113483283660800000000.0;
    }
}

DMat like(Context& ctx, const DMat& a) { return DMat(ctx, a.rows, a.cols, a.cplx, "an exponential work matrix"); }

DMat product(Context& ctx, const DMat& x, const DMat& y) {
    DMat r = like(ctx, x);
    GemmProblem p = make_gemm(x, y, r, 1.0, 0.0, 0.0, 0.0);
    gemm(ctx, p, x.cplx);
    return r;
}

// Ell, :416-430
int ell(Context& ctx, const DMat& a, int m) {
    double a_norm = norm1(ctx, a);
    if (a_norm == 0.0) return 0;
    double apn = one_norm_abs_power(ctx, a, 2 * m + 1);
    if (apn == 0.0) return 0;
    double alpha = apn / (a_norm * abs_coeff_reciprocal(m));
    int value = (int)std::ceil(std::log2(alpha / kUnitRoundoff) / (2 * m));
    return std::max(value, 0);
}

double power_norm(Context& ctx, const DMat& a, int p) {
    NormestResult r = normest_power(ctx, a, p, 2, 5, kSeed);
    return r.value;
}

// SolvePade, :372-405
void solve_pade(Context& ctx, const DMat& u, const DMat& v, DMat& out) {
    int n = u.rows;
    DMat den = like(ctx, u);
    DMat num = like(ctx, u);
    pade_split(ctx, den, num, v, u);
    DBuf piv(ctx, sizeof(int) * (size_t)n);
    LuResult lu = getrf(ctx, den, n, n, 0, piv.as<int>());
    if (lu.singular_column >= 0)
        fail(TNS_E_SINGULAR, "The Pade denominator is exactly singular at column " + std::to_string(lu.singular_column) +
                                 ", which indicates a non-finite input rather than a property of the algorithm.");
    getrs(ctx, den, piv.as<int>(), num, n, false);
    out = std::move(num);
}

// EvaluateLowDegree, :284-315
void evaluate_low(Context& ctx, const double* b, int m, const DMat& a, const DMat& a2, const DMat& a4, const DMat& a6,
                  const DMat* a8, DMat& out) {
    DMat w = like(ctx, a);
    set_identity(ctx, w, b[1]);
    add_scaled(ctx, w, a2, b[3]);
    if (m >= 5) add_scaled(ctx, w, a4, b[5]);
    if (m >= 7) add_scaled(ctx, w, a6, b[7]);
    if (m >= 9) add_scaled(ctx, w, *a8, b[9]);
    DMat u = product(ctx, a, w);
    DMat v = like(ctx, a);
    set_identity(ctx, v, b[0]);
    add_scaled(ctx, v, a2, b[2]);
    if (m >= 5) add_scaled(ctx, v, a4, b[4]);
    if (m >= 7) add_scaled(ctx, v, a6, b[6]);
    if (m >= 9) add_scaled(ctx, v, *a8, b[8]);
    solve_pade(ctx, u, v, out);
}

// EvaluateDegree13, :323-360
void evaluate13(Context& ctx, const DMat& a, const DMat& a2, const DMat& a4, const DMat& a6, DMat& out) {
    const double* b = kPade13;
    DMat inner = like(ctx, a);
    scaled_copy(ctx, inner, a6, b[13]);
    add_scaled(ctx, inner, a4, b[11]);
    add_scaled(ctx, inner, a2, b[9]);
    DMat w = like(ctx, a);
    set_identity(ctx, w, b[1]);
    add_scaled(ctx, w, a2, b[3]);
    add_scaled(ctx, w, a4, b[5]);
    add_scaled(ctx, w, a6, b[7]);
    {
        GemmProblem p = make_gemm(a6, inner, w, 1.0, 0.0, 1.0, 0.0);
        gemm(ctx, p, a.cplx);
    }
    DMat u = product(ctx, a, w);
    DMat inner_even = like(ctx, a);
    scaled_copy(ctx, inner_even, a6, b[12]);
    add_scaled(ctx, inner_even, a4, b[10]);
    add_scaled(ctx, inner_even, a2, b[8]);
    DMat v = like(ctx, a);
    set_identity(ctx, v, b[0]);
    add_scaled(ctx, v, a2, b[2]);
    add_scaled(ctx, v, a4, b[4]);
    add_scaled(ctx, v, a6, b[6]);
    {
        GemmProblem p = make_gemm(a6, inner_even, v, 1.0, 0.0, 1.0, 0.0);
        gemm(ctx, p, a.cplx);
    }
    solve_pade(ctx, u, v, out);
}

// Expmv tables, src/Tensile/MatrixExponentialAction.cs:55-88.
const int kDegrees[] = {1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, 16, 17, 18,
                        19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 35, 40, 45, 50, 55};
const double kThetas[] = {2.29e-16, 2.58e-8, 1.39e-5, 3.40e-4, 2.40e-3, 9.07e-3, 2.38e-2, 5.00e-2, 8.96e-2,
                          1.44e-1,  2.14e-1, 3.00e-1, 4.00e-1, 5.14e-1, 6.41e-1, 7.81e-1, 9.31e-1, 1.09,
                          1.26,     1.44,    1.62,    1.82,    2.01,    2.22,    2.43,    2.64,    2.86,
                          3.08,     3.31,    3.54,    4.7,     6.0,     7.2,     8.5,     9.9};
constexpr int kNumDegrees = 35, kMaxDegree = 55, kMaxPower = 8, kEllProbe = 2;

}  // namespace

// ---------------------------------------------------------------------------

NormestResult normest_power(Context& ctx, const DMat& a, int power, int t, int itmax, int seed) {
    int n = a.rows;
    if (n == 0) return {};
    int tt = std::clamp(t, 1, n);
    if (a.cplx) {
        PowerProbe<CplxE> op(ctx, a, power, tt);
        return estimate<CplxE>(op, n, t, itmax, seed);
    }
    PowerProbe<RealE> op(ctx, a, power, tt);
    return estimate<RealE>(op, n, t, itmax, seed);
}

NormestResult normest_lu_inverse(Context& ctx, const DMat& lu, const int* d_piv, int t, int itmax, int seed) {
    int n = lu.rows;
    if (n == 0) return {};
    int tt = std::clamp(t, 1, n);
    if (lu.cplx) {
        LuInverseProbe<CplxE> op(ctx, lu, d_piv, tt);
        return estimate<CplxE>(op, n, t, itmax, seed);
    }
    LuInverseProbe<RealE> op(ctx, lu, d_piv, tt);
    return estimate<RealE>(op, n, t, itmax, seed);
}

// ScalingAndSquaring, src/Tensile/MatrixExponential.cs:181-270. n >= 2.
void expm(Context& ctx, const DMat& a, DMat& result, ExpmInfo* info) {
    ExpmInfo local;
    if (!info) info = &local;
    *info = ExpmInfo{};
    DMat a2 = product(ctx, a, a);
    DMat a4 = product(ctx, a2, a2);
    DMat a6 = product(ctx, a2, a4);
    double d4 = std::pow(norm1(ctx, a4), 1.0 / 4.0);
    double d6 = std::pow(norm1(ctx, a6), 1.0 / 6.0);
    double eta1 = net::max(d4, d6);
    if (eta1 < kTheta3 && ell(ctx, a, 3) == 0) {
        info->degree = 3;
        evaluate_low(ctx, kPade3, 3, a, a2, a4, a6, nullptr, result);
        return;
    }
    if (eta1 < kTheta5 && ell(ctx, a, 5) == 0) {
        info->degree = 5;
        evaluate_low(ctx, kPade5, 5, a, a2, a4, a6, nullptr, result);
        return;
    }
    double d8 = std::pow(power_norm(ctx, a, 8), 1.0 / 8.0);
    double eta3 = net::max(d6, d8);
    if (eta3 < kTheta7 && ell(ctx, a, 7) == 0) {
        info->degree = 7;
        evaluate_low(ctx, kPade7, 7, a, a2, a4, a6, nullptr, result);
        return;
    }
    if (eta3 < kTheta9 && ell(ctx, a, 9) == 0) {
        info->degree = 9;
        DMat a8 = product(ctx, a4, a4);
        evaluate_low(ctx, kPade9, 9, a, a2, a4, a6, &a8, result);
        return;
    }
    double d10 = std::pow(power_norm(ctx, a, 10), 1.0 / 10.0);
    double eta4 = net::max(d8, d10);
    double eta5 = net::min(eta3, eta4);
    int s = eta5 == 0.0 ? 0 : std::max((int)std::ceil(std::log2(eta5 / kScalingThreshold)), 0);
    {
        DMat sc = like(ctx, a);
        scaled_copy(ctx, sc, a, std::ldexp(1.0, -s));
        s += ell(ctx, sc, 13);
    }
    double factor = std::ldexp(1.0, -s);
    DMat b = like(ctx, a), b2 = like(ctx, a), b4 = like(ctx, a), b6 = like(ctx, a);
    scaled_copy(ctx, b, a, factor);
    scaled_copy(ctx, b2, a2, factor * factor);
    scaled_copy(ctx, b4, a4, std::pow(factor, 4));
    scaled_copy(ctx, b6, a6, std::pow(factor, 6));
    // The powers are no longer needed; give their memory back before the
    // evaluation allocates.
    a2 = DMat();
    a4 = DMat();
    a6 = DMat();
    info->degree = 13;
    info->squarings = s;
    DMat x;
    evaluate13(ctx, b, b2, b4, b6, x);
    DMat sq = like(ctx, a);
    for (int i = 0; i < s; ++i) {
        GemmProblem p = make_gemm(x, x, sq, 1.0, 0.0, 0.0, 0.0);
        gemm(ctx, p, a.cplx);
        std::swap(x, sq);
    }
    result = std::move(x);
}

// MatrixExponentialAction.Dense + Run + SelectParameters,
// src/Tensile/MatrixExponentialAction.cs:149-178, 239-410 (trace shift at the
// typed entry points :138-141 and MatrixExponentialAction.Complex.cs:57-61).
void expmv(Context& ctx, const DMat& a, const DMat& b, double t, DMat& result, ExpmvInfo* info) {
    ExpmvInfo local;
    if (!info) info = &local;
    *info = ExpmvInfo{};
    const int n = a.rows, cols = b.cols;
    const bool cplx = a.cplx;
    // mu = trace / n, per part for complex.
    double tr_re, tr_im;
    trace(ctx, a, &tr_re, &tr_im);
    double mu_re = tr_re / n, mu_im = cplx ? tr_im / n : 0.0;
    DMat sh = like(ctx, a);
    copy_dmat(ctx, sh, a);
    // result[i,i] += -mu: the reference adds the negated shift.
    shift_diagonal(ctx, sh, -mu_re, cplx ? -mu_im : 0.0);
    double one_norm = norm1(ctx, sh);

    double d[kMaxPower + 2];
    for (double& v : d) v = std::numeric_limits<double>::quiet_NaN();
    auto D = [&](int p) {
        if (std::isnan(d[p])) d[p] = std::pow(normest_power(ctx, sh, p, kEllProbe, 5, kSeed).value, 1.0 / p);
        return d[p];
    };
    auto alpha = [&](int p) { return net::max(D(p), D(p + 1)); };

    double scale = std::fabs(t);
    double scaled_norm = scale * one_norm;
    int m = 0, s = 1;
    if (scaled_norm != 0.0) {
        int best_degree = 0;
        double best_scaling = 0.0, best_cost = std::numeric_limits<double>::infinity();
        auto consider = [&](int index, double norm) {
            double scaling = std::ceil(norm / kThetas[index]);
            double cost = kDegrees[index] * scaling;
            if (cost >= best_cost) return;
            best_cost = cost;
            best_degree = kDegrees[index];
            best_scaling = scaling;
        };
        double ca = 2.0 * kEllProbe * kMaxPower * (kMaxPower + 3);
        double cb = kThetas[kNumDegrees - 1] / (cols * (double)kMaxDegree);
        if (scaled_norm <= ca * cb) {
            for (int index = 0; index < kNumDegrees; ++index) consider(index, scaled_norm);
        } else {
            for (int p = 2; p <= kMaxPower; ++p) {
                double alpha_p = scale * alpha(p);
                for (int index = 0; index < kNumDegrees; ++index) {
                    if (kDegrees[index] < (p * (p - 1)) - 1) continue;
                    consider(index, alpha_p);
                }
            }
        }
        double steps = std::max(best_scaling, 1.0);
        if (!std::isfinite(best_cost) || steps > 2147483647.0)
            fail(TNS_E_OUT_OF_RANGE, "||tA||_1 would need more operator applications than this method can finish. "
                                     "Reduce t, or shift the operator.");
        m = best_degree;
        s = (int)steps;
    }
    info->degree = m;
    info->scaling = s;

    DMat f = like(ctx, b), work = like(ctx, b), next = like(ctx, b);
    copy_dmat(ctx, f, b);
    copy_dmat(ctx, work, b);
    // eta = exp(t*mu/s): real (mu*t)/s; complex Complex(mu.re*t, mu.im*t) / (s + 0i).
    double eta_re, eta_im = 0.0;
    if (!cplx) {
        eta_re = std::exp((mu_re * t) / (double)s);
    } else {
        net::Cx e = net::exp(net::div(net::Cx{mu_re * t, mu_im * t}, net::Cx{(double)s, 0.0}));
        eta_re = e.re;
        eta_im = e.im;
    }
    // Panel product on the padded b layout: x and y are (n x cols) with ld rows_p.
    const int ldb = b.ld();
    for (int i = 0; i < s; ++i) {
        double c1 = norminf(ctx, work);
        for (int j = 0; j < m; ++j) {
            double coefficient = t / (s * (double)(j + 1));
            panel_product(ctx, sh, work.p, ldb, next.p, ldb, cols, false);
            scaled_copy(ctx, work, next, coefficient);
            double c2 = norminf(ctx, work);
            add_scaled(ctx, f, work, 1.0);
            info->applications++;
            if (c1 + c2 <= kUnitRoundoff * norminf(ctx, f)) {
                info->early_exits++;
                break;
            }
            c1 = c2;
        }
        if (!(eta_re == 1.0 && eta_im == 0.0)) scale_inplace(ctx, f.p, f.rows_p, f.cols_p, f.ld(), cplx, eta_re, eta_im);
        copy_dmat(ctx, work, f);
    }
    result = std::move(f);
}

}  // namespace tns
