// Al-Mohy & Higham 2009 scaling and squaring (MatrixExponential.ScalingAndSquaring,
// src/Tensile/MatrixExponential.cs:181-270) for a batch of independent
// matrices of any orders, one launch per phase.
//
// Every matrix takes exactly the decisions the reference takes for it: the
// Pade degree ladder (3, 5, 7, 9 against eta1/eta3 and the ell test, then 13),
// d8/d10 from its own normest1 run, s = max(ceil(log2(eta5/4.25)), 0) plus
// ell on the scaled matrix. What is batched is the work between decisions:
// the powers A^2, A^4, A^6 are three grouped GEMM launches for the whole
// batch; the norms, the ell chains and every normest1 product step are one
// launch each for all matrices in that stage; the Pade evaluation is one
// fused elementwise launch and three grouped GEMMs; the LU of the denominators
// advances all matrices block step by block step; the solve and each round
// of squarings are grouped GEMMs over the matrices still squaring. A single
// matrix is a batch of one.
//
// In the split form (Context::split_moduli > 0) every product runs on the
// split product. d4 and d6 then carry intervals that hold the reference's
// values (its FP64 rounding included), and a matrix whose next decision is
// not settled on them has A^2, A^4, A^6 recomputed as the reference computes
// them (powers / make_exact below), so the degree and s stay the reference's.

#include "estimator.h"
#include "pade.h"
#include "tns_internal.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

namespace tns {

namespace {

// Constants, src/Tensile/MatrixExponential.cs:50-110, 441-449 (the Pade
// coefficients are in pade.h).
const double kTheta3 = 1.495585217958292e-2;
const double kTheta5 = 2.539398330063230e-1;
const double kTheta7 = 9.504178996162932e-1;
const double kTheta9 = 2.097847961257068e0;
const double kScalingThreshold = 4.25;
const double kUnitRoundoff = 1.1102230246251565e-16;
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

struct Job {
    const DMat* a = nullptr;
    int n = 0;
    DMat a2, a4, a6, a8;
    double d4 = 0, d6 = 0, d8 = 0, d10 = 0, eta1 = 0, eta3 = 0;
    int degree = 0, s = 0;
    DMat result;
    // Split form: A^2, A^4, A^6 from the split product, with intervals that
    // hold the reference's d4 and d6 (exact: the reference's own products).
    bool exact = true;
    double d4_lo = 0, d4_hi = 0, d6_lo = 0, d6_hi = 0;
};

// An interval [lo, hi] that holds a value the reference computes.
struct Iv {
    double lo, hi;
};
Iv point(double x) { return {x, x}; }
Iv iv_max(Iv a, Iv b) { return {net::max(a.lo, b.lo), net::max(a.hi, b.hi)}; }
Iv iv_min(Iv a, Iv b) { return {net::min(a.lo, b.lo), net::min(a.hi, b.hi)}; }
// Whether x < theta has one answer over the whole interval.
bool certain_below(Iv x, double theta) { return x.hi < theta || x.lo >= theta; }

DMat like(Context& ctx, const DMat& a) { return DMat(ctx, a.rows, a.cols, a.cplx, "an exponential work matrix"); }

// Ell (:416-430) for a set of matrices at one Pade degree m.
std::vector<int> ell_batch(Context& ctx, const std::vector<const DMat*>& mats, int m) {
    std::vector<int> out(mats.size(), 0);
    if (mats.empty()) return out;
    std::vector<double> anorm = norm1_batch(ctx, mats);
    std::vector<double> apn = abs_power_batch(ctx, mats, 2 * m + 1);
    for (size_t k = 0; k < mats.size(); ++k) {
        if (anorm[k] == 0.0 || apn[k] == 0.0) continue;
        double alpha = apn[k] / (anorm[k] * abs_coeff_reciprocal(m));
        int value = (int)std::ceil(std::log2(alpha / kUnitRoundoff) / (2 * m));
        out[k] = std::max(value, 0);
    }
    return out;
}

// normest1 of A_k^p_k (t = 2, itmax = 5, the default seed) for a set of
// (matrix, power) items: every estimator's products of one round run in one
// launch per power step (items of a lower power drop out of the later steps).
template <class TE>
std::vector<double> power_estimates(Context& ctx, const std::vector<const DMat*>& mats,
                                    const std::vector<int>& powers) {
    using Est = Estimator<TE>;
    const size_t cnt = mats.size();
    std::vector<double> out(cnt, 0.0);
    if (cnt == 0) return out;
    std::vector<std::unique_ptr<Est>> est;
    std::vector<size_t> offs(cnt);
    size_t total = 0;
    for (size_t k = 0; k < cnt; ++k) {
        est.emplace_back(new Est(mats[k]->rows, 2, 5, kSeed));
        offs[k] = total;
        total += (size_t)mats[k]->rows * est[k]->t() * TE::kDoubles;
    }
    DBuf d0(ctx, sizeof(double) * std::max<size_t>(total, 1));
    DBuf d1(ctx, sizeof(double) * std::max<size_t>(total, 1));
    std::vector<double> host(total);
    const bool cplx = TE::kDoubles == 2;
    for (;;) {
        for (int phase = 0; phase < 2; ++phase) {
            const bool adjoint = phase == 1;
            std::vector<size_t> live;
            for (size_t k = 0; k < cnt; ++k)
                if (est[k]->need() == (adjoint ? Est::kAdjoint : Est::kApply)) live.push_back(k);
            if (live.empty()) continue;
            for (size_t k : live) {
                const double* src = reinterpret_cast<const double*>(adjoint ? est[k]->s() : est[k]->x());
                std::copy(src, src + (size_t)mats[k]->rows * est[k]->t() * TE::kDoubles, host.data() + offs[k]);
            }
            TNS_CUDA(cudaMemcpyAsync(d0.p, host.data(), sizeof(double) * total, cudaMemcpyHostToDevice, ctx.stream));
            // Each item ping-pongs between its slots of the two buffers; after
            // an odd number of steps its result is in d1.
            int maxp = 0;
            for (size_t k : live) maxp = std::max(maxp, powers[k]);
            for (int step = 0; step < maxp; ++step) {
                double* src = (step % 2 == 0) ? d0.as<double>() : d1.as<double>();
                double* dst = (step % 2 == 0) ? d1.as<double>() : d0.as<double>();
                std::vector<PanelDesc> v;
                for (size_t k : live) {
                    if (powers[k] <= step) continue;
                    int n = mats[k]->rows;
                    v.push_back(PanelDesc{mats[k]->p, n, mats[k]->ld(), src + offs[k], n, dst + offs[k], n, est[k]->t()});
                }
                panel_product_batch(ctx, v, cplx, adjoint);
            }
            TNS_CUDA(cudaMemcpyAsync(host.data(), d0.p, sizeof(double) * total, cudaMemcpyDeviceToHost, ctx.stream));
            std::vector<double> odd(total);
            TNS_CUDA(cudaMemcpyAsync(odd.data(), d1.p, sizeof(double) * total, cudaMemcpyDeviceToHost, ctx.stream));
            ctx.sync();
            for (size_t k : live) {
                double* dstp = reinterpret_cast<double*>(adjoint ? est[k]->z() : est[k]->y());
                const double* from = (powers[k] % 2 == 0 ? host.data() : odd.data()) + offs[k];
                std::copy(from, from + (size_t)mats[k]->rows * est[k]->t() * TE::kDoubles, dstp);
                if (adjoint) est[k]->adjointed();
                else est[k]->applied();
            }
        }
        bool done = true;
        for (auto& e : est)
            if (e->need() != Est::kDone) done = false;
        if (done) break;
    }
    for (size_t k = 0; k < cnt; ++k) out[k] = est[k]->value();
    return out;
}

std::vector<double> power_norms(Context& ctx, const std::vector<const DMat*>& mats, const std::vector<int>& powers) {
    if (mats.empty()) return {};
    return mats[0]->cplx ? power_estimates<CplxE>(ctx, mats, powers) : power_estimates<RealE>(ctx, mats, powers);
}

std::vector<double> power_norms(Context& ctx, const std::vector<const DMat*>& mats, int power) {
    return power_norms(ctx, mats, std::vector<int>(mats.size(), power));
}

// Whether a product may take the split-precision form when the context asks
// for it: the powers that feed the degree and s decisions (A^2, A^4, A^6)
// never do; the Pade evaluation and the squarings may.
enum class Form { kExact, kSplittable };

void product_batch(Context& ctx, std::vector<std::pair<const DMat*, const DMat*>> ab, std::vector<DMat*> c,
                   double beta, Form form = Form::kExact) {
    if (ab.empty()) return;
    if (form == Form::kSplittable && ctx.split_moduli > 0) {
        std::vector<SplitProduct> v;
        for (size_t k = 0; k < ab.size(); ++k) v.push_back(SplitProduct{ab[k].first, ab[k].second, c[k], beta});
        gemm_split_batch(ctx, v, ctx.split_moduli);
        return;
    }
    std::vector<GemmProblem> probs;
    for (size_t k = 0; k < ab.size(); ++k) probs.push_back(make_gemm(*ab[k].first, *ab[k].second, *c[k], 1.0, 0.0, beta, 0.0));
    gemm_grouped(ctx, probs, ab[0].first->cplx);
}

}  // namespace

std::vector<double> power_norm_estimates(Context& ctx, const std::vector<const DMat*>& mats,
                                         const std::vector<int>& powers) {
    return power_norms(ctx, mats, powers);
}

void expm_batch(Context& ctx, const std::vector<const DMat*>& inputs, std::vector<DMat>& results,
                std::vector<ExpmInfo>& infos, const std::function<void(size_t, DMat&&)>& on_final) {
    const size_t cnt = inputs.size();
    results.clear();
    results.resize(cnt);
    infos.assign(cnt, ExpmInfo{});
    if (cnt == 0) return;
    std::vector<Job> jobs(cnt);
    for (size_t k = 0; k < cnt; ++k) {
        jobs[k].a = inputs[k];
        jobs[k].n = inputs[k]->rows;
    }
    // A^2, A^4, A^6 (:190-192) and d4, d6 (:198-199). The split form takes
    // the products from the split product and bounds the reference's d4 and
    // d6 (below); the plain form computes them as the reference does.
    auto powers = [&](std::vector<Job*>& js, Form form) {
        std::vector<std::pair<const DMat*, const DMat*>> ab;
        std::vector<DMat*> c;
        for (auto* j : js) {
            j->a2 = like(ctx, *j->a);
            ab.push_back({j->a, j->a});
            c.push_back(&j->a2);
        }
        product_batch(ctx, ab, c, 0.0, form);
        ab.clear();
        c.clear();
        for (auto* j : js) {
            j->a4 = like(ctx, *j->a);
            ab.push_back({&j->a2, &j->a2});
            c.push_back(&j->a4);
        }
        product_batch(ctx, ab, c, 0.0, form);
        ab.clear();
        c.clear();
        for (auto* j : js) {
            j->a6 = like(ctx, *j->a);
            ab.push_back({&j->a2, &j->a4});
            c.push_back(&j->a6);
        }
        product_batch(ctx, ab, c, 0.0, form);
        std::vector<const DMat*> m4, m6;
        for (auto* j : js) {
            m4.push_back(&j->a4);
            m6.push_back(&j->a6);
        }
        std::vector<double> n4 = norm1_batch(ctx, m4), n6 = norm1_batch(ctx, m6);
        for (size_t k = 0; k < js.size(); ++k) {
            Job& j = *js[k];
            j.d4 = std::pow(n4[k], 1.0 / 4.0);
            j.d6 = std::pow(n6[k], 1.0 / 6.0);
            j.eta1 = net::max(j.d4, j.d6);
            j.exact = form == Form::kExact;
            j.d4_lo = j.d4_hi = j.d4;
            j.d6_lo = j.d6_hi = j.d6;
        }
        if (form == Form::kExact) return;
        // Bounds on |X_ref - X_split|_1 for X = A^2, A^4, A^6, where X_ref is
        // the reference's FP64 product. An FP64 product deviates from the
        // exact one by at most gamma_n |X||Y| entrywise in any summation
        // order, 2 gamma_2n in modulus for the complex 4M product; with
        // |(|X||Y|)|_1 <= |X|_1 |Y|_1 that is g |X|_1 |Y|_1 with g = 4 gamma_n
        // covering both. The split product's own error, about n 2^-t of the
        // same scale, is far inside; the 1-norms' own sums add g of the norm.
        // The widths carry a further factor 2.
        std::vector<const DMat*> m1, m2;
        for (auto* j : js) {
            m1.push_back(j->a);
            m2.push_back(&j->a2);
        }
        std::vector<double> n1 = norm1_batch(ctx, m1), n2 = norm1_batch(ctx, m2);
        for (size_t k = 0; k < js.size(); ++k) {
            Job& j = *js[k];
            const double un = (double)j.n * 1.1102230246251565e-16;
            const double g = 4.0 * un / (1.0 - un);
            const double a1 = n1[k], p2 = n2[k], p4 = n4[k], p6 = n6[k];
            const double e2 = g * a1 * a1;
            const double q2 = p2 + e2;
            const double e4 = g * q2 * q2 + 2.0 * q2 * e2 + e2 * e2;
            const double q4 = p4 + e4;
            const double e6 = g * q2 * q4 + q2 * e4 + e2 * q4 + e2 * e4;
            const double w4 = 2.0 * (e4 + g * p4), w6 = 2.0 * (e6 + g * p6);  // safety factor 2
            j.d4_lo = std::pow(std::max(0.0, p4 - w4), 1.0 / 4.0);
            j.d4_hi = std::pow(p4 + w4, 1.0 / 4.0);
            j.d6_lo = std::pow(std::max(0.0, p6 - w6), 1.0 / 6.0);
            j.d6_hi = std::pow(p6 + w6, 1.0 / 6.0);
        }
    };
    std::vector<Job*> all;
    for (auto& j : jobs) all.push_back(&j);
    powers(all, ctx.split_moduli > 0 ? Form::kSplittable : Form::kExact);
    // Jobs whose next decision could differ from the reference's on the
    // intervals: their powers again, exactly (the reference's arithmetic).
    auto make_exact = [&](std::vector<Job*>& js) {
        if (js.empty()) return;
        powers(js, Form::kExact);
        for (auto* j : js)
            if (j->d8 > 0.0 || j->degree == 0) j->eta3 = net::max(j->d6, j->d8);
        ctx.exact_fallbacks += (long long)js.size();
    };
    auto eta1_iv = [](const Job& j) { return iv_max(Iv{j.d4_lo, j.d4_hi}, Iv{j.d6_lo, j.d6_hi}); };
    auto settle_eta1 = [&](double theta) {
        std::vector<Job*> js;
        for (auto& j : jobs)
            if (j.degree == 0 && !j.exact && !certain_below(eta1_iv(j), theta)) js.push_back(&j);
        make_exact(js);
    };
    // The low-degree ladder (:202-231), stage by stage over the undecided.
    auto stage_ell = [&](int m, auto&& eligible) {
        std::vector<Job*> js;
        std::vector<const DMat*> mats;
        for (auto& j : jobs)
            if (j.degree == 0 && eligible(j)) {
                js.push_back(&j);
                mats.push_back(j.a);
            }
        std::vector<int> e = ell_batch(ctx, mats, m);
        for (size_t k = 0; k < js.size(); ++k)
            if (e[k] == 0) js[k]->degree = m;
    };
    settle_eta1(kTheta3);
    stage_ell(3, [](const Job& j) { return j.eta1 < kTheta3; });
    settle_eta1(kTheta5);
    stage_ell(5, [](const Job& j) { return j.eta1 < kTheta5; });
    {
        std::vector<Job*> js;
        std::vector<const DMat*> mats;
        for (auto& j : jobs)
            if (j.degree == 0) {
                js.push_back(&j);
                mats.push_back(j.a);
            }
        std::vector<double> e8 = power_norms(ctx, mats, 8);
        for (size_t k = 0; k < js.size(); ++k) {
            js[k]->d8 = std::pow(e8[k], 1.0 / 8.0);
            js[k]->eta3 = net::max(js[k]->d6, js[k]->d8);
        }
    }
    auto eta3_iv = [](const Job& j) { return iv_max(Iv{j.d6_lo, j.d6_hi}, point(j.d8)); };
    auto settle_eta3 = [&](double theta) {
        std::vector<Job*> js;
        for (auto& j : jobs)
            if (j.degree == 0 && !j.exact && !certain_below(eta3_iv(j), theta)) js.push_back(&j);
        make_exact(js);
    };
    settle_eta3(kTheta7);
    stage_ell(7, [](const Job& j) { return j.eta3 < kTheta7; });
    settle_eta3(kTheta9);
    stage_ell(9, [](const Job& j) { return j.eta3 < kTheta9; });
    // Degree 13: d10, eta5, s and the ell correction on the scaled matrix (:233-247).
    std::vector<Job*> top;
    for (auto& j : jobs)
        if (j.degree == 0) top.push_back(&j);
    if (!top.empty()) {
        std::vector<const DMat*> mats;
        for (auto* j : top) mats.push_back(j->a);
        std::vector<double> e10 = power_norms(ctx, mats, 10);
        for (size_t k = 0; k < top.size(); ++k) top[k]->d10 = std::pow(e10[k], 1.0 / 10.0);
        {
            // s = max(ceil(log2(eta5 / 4.25)), 0) is monotone in eta5: it is
            // settled when both ends of eta5's interval give the same s.
            auto s_of = [](double eta5) {
                return eta5 == 0.0 ? 0 : std::max((int)std::ceil(std::log2(eta5 / kScalingThreshold)), 0);
            };
            std::vector<Job*> js;
            for (auto* j : top) {
                if (j->exact) continue;
                const Iv e5 = iv_min(eta3_iv(*j), point(net::max(j->d8, j->d10)));
                if (s_of(e5.lo) != s_of(e5.hi)) js.push_back(j);
            }
            make_exact(js);
        }
        std::vector<DMat> scaled;
        std::vector<EwDesc> ew;
        scaled.reserve(top.size());
        for (size_t k = 0; k < top.size(); ++k) {
            Job& j = *top[k];
            double eta4 = net::max(j.d8, j.d10);
            double eta5 = net::min(j.eta3, eta4);
            j.s = eta5 == 0.0 ? 0 : std::max((int)std::ceil(std::log2(eta5 / kScalingThreshold)), 0);
            j.degree = 13;
            scaled.push_back(like(ctx, *j.a));
            ew.push_back(ew_scaled_copy(scaled.back(), *j.a, std::ldexp(1.0, -j.s)));
        }
        ew_batch(ctx, ew);
        std::vector<const DMat*> sm;
        for (auto& m : scaled) sm.push_back(&m);
        std::vector<int> e13 = ell_batch(ctx, sm, 13);
        for (size_t k = 0; k < top.size(); ++k) top[k]->s += e13[k];
    }

    // Evaluation (:251-259, EvaluateLowDegree :284-315, EvaluateDegree13 :323-360).
    // Per job: u (numerator odd part times A) and v (even part); then
    // den = v - u, num = v + u.
    struct Eval {
        DMat b, b6, inner, inner_even, w, u, v;
    };
    std::vector<Eval> ev(cnt);
    {
        // A^8 for degree 9 (:229).
        std::vector<std::pair<const DMat*, const DMat*>> ab;
        std::vector<DMat*> c;
        for (auto& j : jobs)
            if (j.degree == 9) {
                j.a8 = like(ctx, *j.a);
                ab.push_back({&j.a4, &j.a4});
                c.push_back(&j.a8);
            }
        product_batch(ctx, ab, c, 0.0, Form::kSplittable);
        // The numerator's parts, one pass for all jobs (blas1.cu).
        std::vector<PadeDesc> pd;
        for (size_t k = 0; k < cnt; ++k) {
            Job& j = jobs[k];
            Eval& e = ev[k];
            e.w = like(ctx, *j.a);
            e.v = like(ctx, *j.a);
            PadeDesc d{};
            d.a = j.a->p;
            d.a2 = j.a2.p;
            d.a4 = j.a4.p;
            d.a6 = j.a6.p;
            d.a8 = j.degree == 9 ? j.a8.p : nullptr;
            d.w = e.w.p;
            d.v = e.v.p;
            d.count = e.w.bytes() / 8;
            d.rows_p = e.w.rows_p;
            d.n = e.w.rows;
            d.cplx = e.w.cplx ? 1 : 0;
            d.degree = j.degree;
            const double* b = pade_coefficients(j.degree);
            for (int q = 0; q <= j.degree; ++q) d.c[q] = b[q];
            if (j.degree == 13) {
                const double f = std::ldexp(1.0, -j.s);
                e.b = like(ctx, *j.a);
                e.b6 = like(ctx, *j.a);
                e.inner = like(ctx, *j.a);
                e.inner_even = like(ctx, *j.a);
                d.b = e.b.p;
                d.b6 = e.b6.p;
                d.inner = e.inner.p;
                d.inner_even = e.inner_even.p;
                d.f = f;
                d.f2 = f * f;
                d.f4 = std::pow(f, 4);
                d.f6 = std::pow(f, 6);
            }
            pd.push_back(d);
        }
        pade_assemble_batch(ctx, pd);
        // The powers of degree-13 jobs are no longer needed.
        for (auto& j : jobs)
            if (j.degree == 13) {
                j.a2 = DMat();
                j.a4 = DMat();
                j.a6 = DMat();
            }
    }
    {
        // w += B6 inner; v += B6 inner_even (degree 13, beta = 1).
        std::vector<std::pair<const DMat*, const DMat*>> ab;
        std::vector<DMat*> c;
        for (size_t k = 0; k < cnt; ++k)
            if (jobs[k].degree == 13) {
                ab.push_back({&ev[k].b6, &ev[k].inner});
                c.push_back(&ev[k].w);
                ab.push_back({&ev[k].b6, &ev[k].inner_even});
                c.push_back(&ev[k].v);
            }
        product_batch(ctx, ab, c, 1.0, Form::kSplittable);
        // u = A w (B w for degree 13).
        ab.clear();
        c.clear();
        for (size_t k = 0; k < cnt; ++k) {
            ev[k].u = like(ctx, *jobs[k].a);
            ab.push_back({jobs[k].degree == 13 ? &ev[k].b : jobs[k].a, &ev[k].w});
            c.push_back(&ev[k].u);
        }
        product_batch(ctx, ab, c, 0.0, Form::kSplittable);
    }
    // SolvePade (:372-405): den = v - u, num = v + u, LU of den, solve.
    std::vector<DMat> den(cnt), num(cnt);
    {
        std::vector<EwDesc> ew;
        for (size_t k = 0; k < cnt; ++k) {
            den[k] = like(ctx, *jobs[k].a);
            num[k] = like(ctx, *jobs[k].a);
            ew.push_back(ew_pade_split(den[k], num[k], ev[k].v, ev[k].u));
        }
        ew_batch(ctx, ew);
        for (auto& e : ev) e = Eval();  // release the evaluation buffers
        for (auto& j : jobs) {
            j.a2 = DMat();
            j.a4 = DMat();
            j.a6 = DMat();
            j.a8 = DMat();
        }
        size_t piv_total = 0;
        for (auto& j : jobs) piv_total += (size_t)j.n;
        DBuf pivs(ctx, sizeof(int) * (piv_total + cnt));
        std::vector<LuItem> lus;
        std::vector<SolveItem> solves;
        size_t po = 0;
        for (size_t k = 0; k < cnt; ++k) {
            int n = jobs[k].n;
            int* piv = pivs.as<int>() + po;
            int* sing = pivs.as<int>() + piv_total + k;
            lus.push_back(LuItem{&den[k], n, n, 0, piv, sing});
            solves.push_back(SolveItem{&den[k], piv, &num[k], n});
            po += (size_t)n;
        }
        getrf_batch(ctx, lus);
        std::vector<int> sing(cnt);
        TNS_CUDA(cudaMemcpyAsync(sing.data(), pivs.as<int>() + piv_total, sizeof(int) * cnt, cudaMemcpyDeviceToHost,
                                 ctx.stream));
        ctx.sync();
        for (size_t k = 0; k < cnt; ++k)
            if (sing[k] != INT_MAX)
                fail(TNS_E_SINGULAR, "The Pade denominator is exactly singular at column " + std::to_string(sing[k]) +
                                         ", which indicates a non-finite input rather than a property of the algorithm.");
        getrs_batch(ctx, solves, false);
    }
    // A result is final after the solve (s = 0) or after its last squaring.
    auto hand_over = [&](int s_done) {
        if (!on_final) return;
        for (size_t k = 0; k < cnt; ++k)
            if (jobs[k].s == s_done) on_final(k, std::move(num[k]));
    };
    hand_over(0);
    // Squarings (:262-267): round r squares every matrix with s > r.
    {
        std::vector<DMat> sq(cnt);
        int max_s = 0;
        for (auto& j : jobs) max_s = std::max(max_s, j.s);
        for (size_t k = 0; k < cnt; ++k)
            if (jobs[k].s > 0) sq[k] = like(ctx, *jobs[k].a);
        for (int r = 0; r < max_s; ++r) {
            std::vector<std::pair<const DMat*, const DMat*>> ab;
            std::vector<DMat*> c;
            for (size_t k = 0; k < cnt; ++k)
                if (jobs[k].s > r) {
                    ab.push_back({&num[k], &num[k]});
                    c.push_back(&sq[k]);
                }
            product_batch(ctx, ab, c, 0.0, Form::kSplittable);
            for (size_t k = 0; k < cnt; ++k)
                if (jobs[k].s > r) std::swap(num[k], sq[k]);
            hand_over(r + 1);
        }
    }
    for (size_t k = 0; k < cnt; ++k) {
        results[k] = std::move(num[k]);
        infos[k].degree = jobs[k].degree;
        infos[k].squarings = jobs[k].degree == 13 ? jobs[k].s : 0;
    }
}

void expm(Context& ctx, const DMat& a, DMat& result, ExpmInfo* info) {
    std::vector<DMat> results;
    std::vector<ExpmInfo> infos;
    expm_batch(ctx, {&a}, results, infos);
    result = std::move(results[0]);
    if (info) *info = infos[0];
}

}  // namespace tns
