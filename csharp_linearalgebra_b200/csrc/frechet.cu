// The Frechet derivative of the matrix exponential and the adjoint of
// exp(tA)B (the differentiation form).
//
// L(A, E) = d/dh exp(A + hE) at h = 0. Tensile has no routine for it; the
// reference's own way to the same quantity is its Expm of the 2n x 2n block
// matrix [[A, E], [0, A]], whose upper right block is L(A, E)
// (MatrixExponential.ScalingAndSquaring, src/Tensile/MatrixExponential.cs:181-270),
// which the tests compare against. Here the derivative is computed at about
// three times the cost of exp(A) instead of eight, by the structured Pade
// scaling-and-squaring algorithm of Al-Mohy and Higham ("Computing the
// Frechet derivative of the matrix exponential, with an application to
// condition number estimation", SIAM J. Matrix Anal. Appl. 30 (2009),
// Algorithm 6.4):
//   - degree m = the first of 3, 5, 7, 9 with ||A||_1 <= l_m, else 13 with
//     s = max(0, ceil(log2(||A||_1 / l_13))), B = 2^-s A, E_s = 2^-s E;
//   - r_m(B) = q(B)^-1 p(B) with p = V + U, q = V - U (U the odd part, V the
//     even part of the numerator), and its derivative
//     L_r = q^-1 (L_U + L_V + (L_U - L_V) r), where L_U, L_V follow from the
//     derivatives of the even powers: M_2 = B E_s + E_s B,
//     M_4 = B^2 M_2 + M_2 B^2, M_6 = B^4 M_2 + M_4 B^2, M_8 = B^4 M_4 + M_4 B^4;
//   - s squarings: L <- X L + L X, X <- X^2.
// The work is split in two passes. The forward pass computes exp(A) and keeps
// what the derivative needs: the scaled powers, the Pade polynomial parts,
// the LU factors of q(B), and the squarings X_0 .. X_s when the device has
// room for them (Context::checkpoint_bytes), else X_0 alone, from which the
// derivative pass squares again. The derivative pass is linear in E and can
// run for any direction after the forward pass.
//
// Adjoint of exp(tA)B. For F = exp(tA) B, loss = ||F - Y||_F^2 and
// G = 2 (F - Y), the gradients (dloss = Re <grad, d.>, <X, Y> = tr(X^H Y)) are
//   dloss/dB = exp(tA)^H G = exp(t A^H) G,
//   dloss/dA = t L(t A^H, G B^H)   (L(X, .) has the adjoint L(X^H, .)),
//   dloss/dt = Re tr(G^H A F).
// One forward pass on t A^H gives exp(tA)^H (hence exp(tA) and F), and one
// derivative pass in the direction G B^H gives dloss/dA.
//
// Every product is the grouped DMMA GEMM in plain FP64; LU and solves are the
// library's own. No integer decision here belongs to the reference, so none
// has to be bit-exact; the tests hold the results to the block Expm and to
// central differences.

#include "pade.h"
#include "tns_internal.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <string>
#include <vector>

namespace tns {

namespace {

// l_m of Al-Mohy and Higham (2009), Table 6.1: the largest ||A||_1 for which
// the degree-m Pade approximant meets the backward error bound of unit
// roundoff for both exp(A) and L(A, E) without scaling.
const double kEll3 = 1.08e-2;
const double kEll5 = 2.00e-1;
const double kEll7 = 7.83e-1;
const double kEll9 = 1.78e0;
const double kEll13 = 4.74e0;

DMat like(Context& ctx, const DMat& a, const char* purpose = "a Frechet work matrix") {
    return DMat(ctx, a.rows, a.cols, a.cplx, purpose);
}

// c := a b + beta c.
void mul(Context& ctx, const DMat& a, const DMat& b, DMat& c, double beta = 0.0) {
    std::vector<GemmProblem> p{make_gemm(a, b, c, 1.0, 0.0, beta, 0.0)};
    gemm_grouped(ctx, p, a.cplx);
}

struct Term {
    double f;
    const DMat* m;  // nullptr: the identity
};
// dst := sum of f * m over the terms, in order; only the first may be the
// identity (it sets dst).
void combine(Context& ctx, DMat& dst, std::initializer_list<Term> terms) {
    bool first = true;
    for (const Term& t : terms) {
        if (!first && !t.m) fail(TNS_E_ARGUMENT, "internal: identity term after the first");
        std::vector<EwDesc> v{first ? (t.m ? ew_scaled_copy(dst, *t.m, t.f) : ew_identity(dst, t.f))
                                    : ew_add_scaled(dst, *t.m, t.f)};
        ew_batch(ctx, v);
        first = false;
    }
}

struct Forward {
    int n = 0, degree = 0, s = 0;
    DMat b, b2, b4, b6, b8;  // B = 2^-s A and its even powers (b8: degree 9)
    DMat w1, z1;             // degree 13: W1 and Z1 of the Pade numerator
    DMat w;                  // U = B w: w = B^6 W1 + W2 (degree 13) or the odd polynomial
    DMat lu;                 // LU factors of q(B) = V - U
    DBuf piv;
    std::vector<DMat> x;     // X_0 .. X_s, or X_0 alone
    DMat result;             // exp(A)
};

void forward(Context& ctx, const DMat& a, Forward& f) {
    const int n = a.rows;
    f.n = n;
    const double nrm = norm1(ctx, a);
    if (!std::isfinite(nrm)) fail(TNS_E_ARGUMENT, "The matrix has a non-finite entry.");
    if (nrm <= kEll3) f.degree = 3;
    else if (nrm <= kEll5) f.degree = 5;
    else if (nrm <= kEll7) f.degree = 7;
    else if (nrm <= kEll9) f.degree = 9;
    else {
        f.degree = 13;
        f.s = std::max(0, (int)std::ceil(std::log2(nrm / kEll13)));
    }
    const int m = f.degree;
    const double* c = pade_coefficients(m);
    f.b = like(ctx, a);
    {
        std::vector<EwDesc> v{ew_scaled_copy(f.b, a, std::ldexp(1.0, -f.s))};
        ew_batch(ctx, v);
    }
    f.b2 = like(ctx, a);
    mul(ctx, f.b, f.b, f.b2);
    if (m >= 5) {
        f.b4 = like(ctx, a);
        mul(ctx, f.b2, f.b2, f.b4);
    }
    if (m >= 7) {
        f.b6 = like(ctx, a);
        mul(ctx, f.b4, f.b2, f.b6);
    }
    if (m == 9) {
        f.b8 = like(ctx, a);
        mul(ctx, f.b4, f.b4, f.b8);
    }
    f.w = like(ctx, a);
    DMat v = like(ctx, a);
    if (m == 13) {
        f.w1 = like(ctx, a);
        f.z1 = like(ctx, a);
        combine(ctx, f.w1, {{c[13], &f.b6}, {c[11], &f.b4}, {c[9], &f.b2}});
        combine(ctx, f.z1, {{c[12], &f.b6}, {c[10], &f.b4}, {c[8], &f.b2}});
        combine(ctx, f.w, {{c[1], nullptr}, {c[3], &f.b2}, {c[5], &f.b4}, {c[7], &f.b6}});
        combine(ctx, v, {{c[0], nullptr}, {c[2], &f.b2}, {c[4], &f.b4}, {c[6], &f.b6}});
        mul(ctx, f.b6, f.w1, f.w, 1.0);
        mul(ctx, f.b6, f.z1, v, 1.0);
    } else {
        const DMat* pw[] = {nullptr, &f.b2, &f.b4, &f.b6, &f.b8};
        std::vector<EwDesc> s1{ew_identity(f.w, c[1]), ew_identity(v, c[0])};
        ew_batch(ctx, s1);
        for (int k = 1; 2 * k <= m - 1; ++k) {
            std::vector<EwDesc> sk{ew_add_scaled(f.w, *pw[k], c[2 * k + 1]), ew_add_scaled(v, *pw[k], c[2 * k])};
            ew_batch(ctx, sk);
        }
    }
    DMat u = like(ctx, a);
    mul(ctx, f.b, f.w, u);
    f.lu = like(ctx, a);
    DMat x0 = like(ctx, a, "the Pade approximant");
    {
        std::vector<EwDesc> sp{ew_pade_split(f.lu, x0, v, u)};
        ew_batch(ctx, sp);
    }
    f.piv = DBuf(ctx, sizeof(int) * (size_t)n);
    LuResult r = getrf(ctx, f.lu, n, n, 0, f.piv.as<int>());
    if (r.singular_column >= 0)
        fail(TNS_E_SINGULAR, "The Pade denominator is exactly singular at column " + std::to_string(r.singular_column) +
                                 ", which indicates a non-finite input rather than a property of the algorithm.");
    getrs(ctx, f.lu, f.piv.as<int>(), x0, n, false);
    // Keep every squaring when the budget allows, else X_0 alone.
    long long budget = ctx.checkpoint_bytes;
    if (budget < 0) {
        size_t free_b = 0, total_b = 0;
        TNS_CUDA(cudaMemGetInfo(&free_b, &total_b));
        budget = (long long)(free_b / 4);
    }
    const bool keep = (long long)x0.bytes() * (f.s + 1) <= budget;
    f.x.clear();
    f.x.push_back(std::move(x0));
    DMat cur;
    for (int k = 1; k <= f.s; ++k) {
        const DMat& prev = keep || k == 1 ? f.x.back() : cur;
        DMat next = like(ctx, a, "a squaring of the Pade approximant");
        mul(ctx, prev, prev, next);
        if (keep) f.x.push_back(std::move(next));
        else cur = std::move(next);
    }
    if (f.s == 0) {
        f.result = like(ctx, a, "exp(A)");
        copy_dmat(ctx, f.result, f.x[0]);
    } else if (keep) {
        f.result = std::move(f.x.back());  // X_s itself is not needed by the derivative
        f.x.pop_back();
    } else {
        f.result = std::move(cur);
    }
}

// l := L(A, E) from the forward pass of A.
void derivative(Context& ctx, const Forward& f, const DMat& e, DMat& l) {
    const int m = f.degree;
    const double* c = pade_coefficients(m);
    DMat es = like(ctx, e);
    {
        std::vector<EwDesc> v{ew_scaled_copy(es, e, std::ldexp(1.0, -f.s))};
        ew_batch(ctx, v);
    }
    DMat m2 = like(ctx, e), m4, m6, m8;
    mul(ctx, f.b, es, m2);
    mul(ctx, es, f.b, m2, 1.0);
    if (m >= 5) {
        m4 = like(ctx, e);
        mul(ctx, f.b2, m2, m4);
        mul(ctx, m2, f.b2, m4, 1.0);
    }
    if (m >= 7) {
        m6 = like(ctx, e);
        mul(ctx, f.b4, m2, m6);
        mul(ctx, m4, f.b2, m6, 1.0);
    }
    if (m == 9) {
        m8 = like(ctx, e);
        mul(ctx, f.b4, m4, m8);
        mul(ctx, m4, f.b4, m8, 1.0);
    }
    DMat lw = like(ctx, e), lv = like(ctx, e);
    if (m == 13) {
        DMat lw1 = like(ctx, e), lz1 = like(ctx, e);
        combine(ctx, lw1, {{c[13], &m6}, {c[11], &m4}, {c[9], &m2}});
        combine(ctx, lz1, {{c[12], &m6}, {c[10], &m4}, {c[8], &m2}});
        combine(ctx, lw, {{c[7], &m6}, {c[5], &m4}, {c[3], &m2}});
        combine(ctx, lv, {{c[6], &m6}, {c[4], &m4}, {c[2], &m2}});
        mul(ctx, f.b6, lw1, lw, 1.0);
        mul(ctx, m6, f.w1, lw, 1.0);
        mul(ctx, f.b6, lz1, lv, 1.0);
        mul(ctx, m6, f.z1, lv, 1.0);
    } else {
        const DMat* md[] = {nullptr, &m2, &m4, &m6, &m8};
        {
            std::vector<EwDesc> s1{ew_scaled_copy(lw, m2, c[3]), ew_scaled_copy(lv, m2, c[2])};
            ew_batch(ctx, s1);
        }
        for (int k = 2; 2 * k <= m - 1; ++k) {
            std::vector<EwDesc> sk{ew_add_scaled(lw, *md[k], c[2 * k + 1]), ew_add_scaled(lv, *md[k], c[2 * k])};
            ew_batch(ctx, sk);
        }
    }
    // L_U = B L_W + E_s W.
    DMat lu = like(ctx, e);
    mul(ctx, f.b, lw, lu);
    mul(ctx, es, f.w, lu, 1.0);
    // rhs = L_U + L_V + (L_U - L_V) X_0; L_0 = q(B)^-1 rhs.
    DMat rhs = like(ctx, e), diff = like(ctx, e);
    {
        std::vector<EwDesc> v{ew_pade_split(diff, rhs, lu, lv)};  // diff = L_U - L_V, rhs = L_U + L_V
        ew_batch(ctx, v);
    }
    mul(ctx, diff, f.x[0], rhs, 1.0);
    getrs(ctx, f.lu, f.piv.as<int>(), rhs, f.n, false);
    // Squarings: L_k = X_{k-1} L_{k-1} + L_{k-1} X_{k-1}.
    const bool kept = (int)f.x.size() >= f.s;
    const DMat* x = &f.x[0];
    DMat cur, tmp;
    DMat next = like(ctx, e);
    for (int k = 1; k <= f.s; ++k) {
        if (kept) x = &f.x[k - 1];
        mul(ctx, *x, rhs, next);
        mul(ctx, rhs, *x, next, 1.0);
        std::swap(rhs, next);
        if (!kept && k < f.s) {
            // X_k for the next step, squared again from X_{k-1}.
            if (tmp.p == nullptr) tmp = like(ctx, e);
            mul(ctx, *x, *x, tmp);
            std::swap(cur, tmp);
            x = &cur;
        }
    }
    l = std::move(rhs);
}

}  // namespace

void expm_frechet(Context& ctx, const DMat& a, const DMat& e, DMat* expa, DMat& l, ExpmInfo* info) {
    if (a.rows != a.cols || e.rows != a.rows || e.cols != a.cols || a.cplx != e.cplx)
        fail(TNS_E_ARGUMENT, "internal Frechet derivative of non-conformable matrices");
    Forward f;
    forward(ctx, a, f);
    derivative(ctx, f, e, l);
    if (expa) *expa = std::move(f.result);
    if (info) {
        info->degree = f.degree;
        info->squarings = f.s;
    }
}

GradientResult expmv_gradient(Context& ctx, const DMat& a, const DMat& b, const DMat& y, double t, DMat* f_out,
                              DMat& grad_a, DMat& grad_b) {
    const int n = a.rows, nc = b.cols;
    const bool cplx = a.cplx;
    if (a.rows != a.cols || b.rows != n || y.rows != n || y.cols != nc || b.cplx != cplx || y.cplx != cplx)
        fail(TNS_E_ARGUMENT, "internal gradient of non-conformable matrices");
    GradientResult res;
    // Forward pass on t A^H: exp(t A^H) = exp(tA)^H.
    DMat ah(ctx, n, n, cplx, "t A^H");
    conj_transpose(ctx, ah, a);
    {
        std::vector<EwDesc> v{ew_scaled_copy(ah, ah, t)};
        ew_batch(ctx, v);
    }
    Forward fw;
    forward(ctx, ah, fw);
    res.info.degree = fw.degree;
    res.info.squarings = fw.s;
    const DMat& xh = fw.result;  // exp(tA)^H
    DMat x(ctx, n, n, cplx, "exp(tA)");
    conj_transpose(ctx, x, xh);
    DMat f(ctx, n, nc, cplx, "exp(tA) B");
    mul(ctx, x, b, f);
    x = DMat();
    // G = 2 (F - Y); loss = ||F - Y||_F^2.
    DMat g(ctx, n, nc, cplx, "the loss gradient with respect to F");
    {
        std::vector<EwDesc> v1{ew_scaled_copy(g, f, 1.0)};
        ew_batch(ctx, v1);
        std::vector<EwDesc> v2{ew_add_scaled(g, y, -1.0)};
        ew_batch(ctx, v2);
    }
    const double r = normfro(ctx, g);
    res.loss = r * r;
    {
        std::vector<EwDesc> v{ew_scaled_copy(g, g, 2.0)};
        ew_batch(ctx, v);
    }
    // dloss/dB = exp(tA)^H G.
    grad_b = DMat(ctx, n, nc, cplx, "the gradient with respect to B");
    mul(ctx, xh, g, grad_b);
    // dloss/dt = Re tr(G^H A F).
    {
        DMat af(ctx, n, nc, cplx, "A exp(tA) B");
        mul(ctx, a, f, af);
        DMat gh(ctx, nc, n, cplx, "G^H");
        conj_transpose(ctx, gh, g);
        DMat small(ctx, nc, nc, cplx, "G^H A F");
        mul(ctx, gh, af, small);
        std::vector<double> host((size_t)small.rows_p * small.cols_p * (cplx ? 2 : 1));
        TNS_CUDA(cudaMemcpyAsync(host.data(), small.p, small.bytes(), cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        double tr = 0.0;
        for (int i = 0; i < nc; ++i) tr += host[((size_t)i * small.rows_p + i) * (cplx ? 2 : 1)];
        res.grad_t = tr;
    }
    // dloss/dA = t L(t A^H, G B^H).
    DMat bh(ctx, nc, n, cplx, "B^H");
    conj_transpose(ctx, bh, b);
    DMat dir(ctx, n, n, cplx, "G B^H");
    mul(ctx, g, bh, dir);
    DMat l;
    derivative(ctx, fw, dir, l);
    grad_a = DMat(ctx, n, n, cplx, "the gradient with respect to A");
    {
        std::vector<EwDesc> v{ew_scaled_copy(grad_a, l, t)};
        ew_batch(ctx, v);
    }
    if (f_out) *f_out = std::move(f);
    return res;
}

}  // namespace tns
