// The reference's whole algorithms on the device, besides Expm
// (expm_batched.cu): the Higham-Tisseur block 1-norm estimator over dense
// power operators and LU inverses, and Al-Mohy & Higham 2011 truncated
// Taylor (Expmv).
//
// Control flow and every scalar decision run on the host in the reference's
// order, with the reference's constants; all O(n^2) and O(n^3) work runs in
// the sm_100a kernels. The estimator's bookkeeping (signs, column norms, the
// sort of candidates) is O(n t) and runs on the host over panels copied back
// from the device; the products run on the device.

#include "estimator.h"
#include "tns_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <limits>
#include <vector>

namespace tns {

namespace {

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
    bool free_order;
    DMat panel;
    LuInverseProbe(Context& c, const DMat& lu_, const int* piv, int t, bool free)
        : ctx(c), lu(lu_), d_piv(piv), free_order(free), panel(c, lu_.rows, t, lu_.cplx, "an estimator probe panel") {}
    void apply(const typename TE::T* x, typename TE::T* y, int t, bool adjoint) override {
        int n = lu.rows;
        size_t esz = sizeof(double) * TE::kDoubles;
        TNS_CUDA(cudaMemcpy2DAsync(panel.p, (size_t)panel.ld() * esz, x, (size_t)n * esz, (size_t)n * esz, t,
                                   cudaMemcpyHostToDevice, ctx.stream));
        if (free_order) getrs_free_order(ctx, lu, d_piv, panel, t, adjoint);
        else getrs(ctx, lu, d_piv, panel, t, adjoint);
        TNS_CUDA(cudaMemcpy2DAsync(y, (size_t)n * esz, panel.p, (size_t)panel.ld() * esz, (size_t)n * esz, t,
                                   cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
    }
};

// An operator given as an in-place device solve on a panel of `rows` rows
// (the probe's n rows, zeros below).
template <class TE>
struct SolveProbe : Probe<TE> {
    Context& ctx;
    int n;
    const std::function<void(DMat&, int, bool)>& solve;
    DMat panel;
    SolveProbe(Context& c, int n_, int rows, bool cplx, const std::function<void(DMat&, int, bool)>& s, int t)
        : ctx(c), n(n_), solve(s), panel(c, rows, t, cplx, "an estimator probe panel") {}
    void apply(const typename TE::T* x, typename TE::T* y, int t, bool adjoint) override {
        const size_t esz = sizeof(double) * TE::kDoubles;
        panel.zero();
        TNS_CUDA(cudaMemcpy2DAsync(panel.p, (size_t)panel.ld() * esz, x, (size_t)n * esz, (size_t)n * esz, t,
                                   cudaMemcpyHostToDevice, ctx.stream));
        solve(panel, t, adjoint);
        TNS_CUDA(cudaMemcpy2DAsync(y, (size_t)n * esz, panel.p, (size_t)panel.ld() * esz, (size_t)n * esz, t,
                                   cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
    }
};

// A caller's operator (IAdjointOperator<T>, src/Tensile/LinearOperators.cs:37-75):
// the probe panel goes to the device, the caller's apply or adjoint callback
// writes the result there on the context's stream, and it comes back.
template <class TE>
struct OperatorProbe : Probe<TE> {
    Context& ctx;
    int n;
    ApplyFn apply_fn, adjoint_fn;
    void* user;
    DMat x, y;
    OperatorProbe(Context& c, int n_, ApplyFn ap, ApplyFn adj, void* u, int t)
        : ctx(c), n(n_), apply_fn(ap), adjoint_fn(adj), user(u), x(c, n_, t, TE::kDoubles == 2, "an estimator probe panel"),
          y(c, n_, t, TE::kDoubles == 2, "an estimator probe panel") {}
    void apply(const typename TE::T* xs, typename TE::T* ys, int t, bool adjoint) override {
        const size_t esz = sizeof(double) * TE::kDoubles;
        TNS_CUDA(cudaMemcpy2DAsync(x.p, (size_t)x.ld() * esz, xs, (size_t)n * esz, (size_t)n * esz, t,
                                   cudaMemcpyHostToDevice, ctx.stream));
        const int rc = (adjoint ? adjoint_fn : apply_fn)(user, t, x.p, y.p, x.ld(), ctx.stream);
        if (rc != 0)
            fail(TNS_E_OPERATOR, std::string("the operator's ") + (adjoint ? "adjoint" : "apply") +
                                     " callback returned " + std::to_string(rc));
        TNS_CUDA(cudaMemcpy2DAsync(ys, (size_t)n * esz, y.p, (size_t)y.ld() * esz, (size_t)n * esz, t,
                                   cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
    }
};

// Drive one estimator to completion through a probe (NormEstimate.Estimate).
template <class TE>
NormestResult estimate(Probe<TE>& op, int n, int columns, int max_iterations, int seed) {
    Estimator<TE> e(n, columns, max_iterations, seed);
    while (e.need() != Estimator<TE>::kDone) {
        if (e.need() == Estimator<TE>::kApply) {
            op.apply(e.x(), e.y(), e.t(), false);
            e.applied();
        } else {
            op.apply(e.s(), e.z(), e.t(), true);
            e.adjointed();
        }
    }
    return {e.value(), e.iterations(), e.products()};
}

const double kUnitRoundoff = 1.1102230246251565e-16;
const int kSeed = 20260915;

DMat like(Context& ctx, const DMat& a) { return DMat(ctx, a.rows, a.cols, a.cplx, "an exponential work matrix"); }

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

NormestResult normest_solve(Context& ctx, int n, int rows, bool cplx,
                            const std::function<void(DMat&, int, bool)>& solve, int t, int itmax, int seed) {
    if (n == 0) return {};
    int tt = std::clamp(t, 1, n);
    if (cplx) {
        SolveProbe<CplxE> op(ctx, n, rows, true, solve, tt);
        return estimate<CplxE>(op, n, t, itmax, seed);
    }
    SolveProbe<RealE> op(ctx, n, rows, false, solve, tt);
    return estimate<RealE>(op, n, t, itmax, seed);
}

NormestResult normest_operator(Context& ctx, int n, bool cplx, ApplyFn apply, ApplyFn adjoint, void* user, int t,
                               int itmax, int seed) {
    if (n == 0) return {};
    int tt = std::clamp(t, 1, n);
    if (cplx) {
        OperatorProbe<CplxE> op(ctx, n, apply, adjoint, user, tt);
        return estimate<CplxE>(op, n, t, itmax, seed);
    }
    OperatorProbe<RealE> op(ctx, n, apply, adjoint, user, tt);
    return estimate<RealE>(op, n, t, itmax, seed);
}

NormestResult normest_lu_inverse(Context& ctx, const DMat& lu, const int* d_piv, int t, int itmax, int seed,
                                 bool free_order) {
    int n = lu.rows;
    if (n == 0) return {};
    int tt = std::clamp(t, 1, n);
    if (lu.cplx) {
        LuInverseProbe<CplxE> op(ctx, lu, d_piv, tt, free_order);
        return estimate<CplxE>(op, n, t, itmax, seed);
    }
    LuInverseProbe<RealE> op(ctx, lu, d_piv, tt, free_order);
    return estimate<RealE>(op, n, t, itmax, seed);
}

// MatrixExponentialAction.Dense + Run + SelectParameters,
// src/Tensile/MatrixExponentialAction.cs:149-178, 239-410 (trace shift at the
// typed entry points :138-141 and MatrixExponentialAction.Complex.cs:57-61).
namespace {

// (m, s) as MatrixExponentialAction.SelectParameters (:347-398): minimise m s
// over the Taylor degrees subject to the backward error bound; below
// condition 3.13, or without the sharp bounds (a matrix-free operator), the
// crude bound from ||tA||_1 over every degree.
void select_parameters(double scaled_norm, const std::function<double(int)>* alpha, double scale, int cols, int& m,
                       int& s) {
    m = 0;
    s = 1;
    if (scaled_norm == 0.0) return;
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
    if (alpha == nullptr || scaled_norm <= ca * cb) {
        for (int index = 0; index < kNumDegrees; ++index) consider(index, scaled_norm);
    } else {
        for (int p = 2; p <= kMaxPower; ++p) {
            double alpha_p = scale * (*alpha)(p);
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

// Run (:239-320): the scaled Taylor recurrence with early exit, over
// y := A x for (n x cols) panels of leading dimension ld in device memory.
void taylor_run(Context& ctx, const std::function<void(const double*, double*, int)>& apply, const DMat& b,
                double t, int m, int s, double eta_re, double eta_im, ExpmvInfo* info, DMat& result) {
    const bool cplx = b.cplx;
    DMat f = like(ctx, b), work = like(ctx, b), next = like(ctx, b);
    copy_dmat(ctx, f, b);
    copy_dmat(ctx, work, b);
    const int ldb = b.ld();
    for (int i = 0; i < s; ++i) {
        double c1 = norminf(ctx, work);
        for (int j = 0; j < m; ++j) {
            double coefficient = t / (s * (double)(j + 1));
            apply(work.p, next.p, ldb);
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

}  // namespace

void expmv_select_parameters(double scaled_norm, const std::function<double(int)>* alpha, double scale, int cols,
                             int& m, int& s) {
    select_parameters(scaled_norm, alpha, scale, cols, m, s);
}

void expmv_taylor_host(Context& ctx, const DMat& shifted, const DMat& b, double t, int m, int s, double eta_re,
                       double eta_im, DMat& result, ExpmvInfo* info) {
    const int cols_b = b.cols;
    taylor_run(
        ctx, [&](const double* x, double* y, int ld) { panel_product(ctx, shifted, x, ld, y, ld, cols_b, false); }, b,
        t, m, s, eta_re, eta_im, info, result);
}

void expmv_host_loop(Context& ctx, const DMat& a, const DMat& b, double t, DMat& result, ExpmvInfo* info) {
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
    const std::function<double(int)> alpha = [&](int p) { return net::max(D(p), D(p + 1)); };

    int m = 0, s = 1;
    select_parameters(std::fabs(t) * one_norm, &alpha, std::fabs(t), cols, m, s);
    info->degree = m;
    info->scaling = s;
    // eta = exp(t*mu/s): real (mu*t)/s; complex Complex(mu.re*t, mu.im*t) / (s + 0i).
    double eta_re, eta_im = 0.0;
    if (!cplx) {
        eta_re = std::exp((mu_re * t) / (double)s);
    } else {
        net::Cx e = net::exp(net::div(net::Cx{mu_re * t, mu_im * t}, net::Cx{(double)s, 0.0}));
        eta_re = e.re;
        eta_im = e.im;
    }
    const int cols_b = b.cols;
    taylor_run(
        ctx, [&](const double* x, double* y, int ld) { panel_product(ctx, sh, x, ld, y, ld, cols_b, false); }, b, t,
        m, s, eta_re, eta_im, info, result);
}

void expmv_operator(Context& ctx, int n, ApplyFn apply, void* user, const DMat& b, double t, double bound,
                    DMat& result, ExpmvInfo* info) {
    ExpmvInfo local;
    if (!info) info = &local;
    *info = ExpmvInfo{};
    if (b.rows != n) fail(TNS_E_ARGUMENT, "B has the wrong number of rows for the operator");
    int m = 0, s = 1;
    select_parameters(std::fabs(t) * bound, nullptr, std::fabs(t), b.cols, m, s);
    info->degree = m;
    info->scaling = s;
    const int cols = b.cols;
    // No trace, so no shift: mu = 0 and eta = 1 (:227-228).
    taylor_run(
        ctx,
        [&](const double* x, double* y, int ld) {
            const int rc = apply(user, cols, x, y, ld, ctx.stream);
            if (rc != 0) fail(TNS_E_OPERATOR, "the operator's apply callback returned " + std::to_string(rc));
        },
        b, t, m, s, 1.0, 0.0, info, result);
}

}  // namespace tns
