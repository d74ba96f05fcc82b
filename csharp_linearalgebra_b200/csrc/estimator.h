// The Higham-Tisseur block 1-norm estimator (NormEstimate.Estimate,
// src/Tensile/NormEstimate.cs:104-274) as a resumable state machine: the
// caller applies the operator (A X, then A^H S) wherever it likes -- one
// matrix at a time, or a whole batch of estimators in one device launch --
// and the bookkeeping between the products is the reference's, step for step,
// with its seeded System.Random and its Array.Sort.
#pragma once

#include <algorithm>
#include <cmath>
#include <vector>

#include "net_compat.h"

namespace tns {

// IElementKernels<T> members the estimator uses (src/Tensile/ElementKernels.cs:137-157,
// src/Tensile/ComplexKernels.cs:111-129).
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
    static T from_real(double v) { return v; }
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
    static T from_real(double v) { return {v, 0.0}; }
};

template <class TE>
class Estimator {
public:
    using T = typename TE::T;
    enum Need { kApply, kAdjoint, kDone };

    Estimator(int n, int columns, int max_iterations, int seed) : n_(n), rng_(seed) {
        if (n == 0) {
            need_ = kDone;
            return;
        }
        t_ = std::clamp(columns, 1, n);
        itmax_ = std::max(max_iterations, 2);
        size_t extent = (size_t)n * t_;
        x_.resize(extent);
        y_.resize(extent);
        s_.resize(extent);
        s_old_.resize(extent);
        z_.resize(extent);
        h_.resize(n);
        keys_.resize(n);
        order_.resize(n);
        scratch_.resize(n);
        current_.resize(t_);
        used_.assign(n, 0);
        // InitialProbe, :281-299: a column of ones, the rest random +/-1
        // distinct from their predecessors, all scaled to unit 1-norm.
        for (int i = 0; i < n; ++i) x_[i] = TE::one();
        for (int j = 1; j < t_; ++j)
            for (int attempt = 0; attempt < 8; ++attempt) {
                fill_signs(x_.data() + (size_t)j * n);
                if (!parallel_to_any(x_.data() + (size_t)j * n, x_.data(), j)) break;
            }
        T scale = TE::from_real(1.0 / n);
        for (size_t i = 0; i < extent; ++i) x_[i] = TE::mul(x_[i], scale);
        need_ = kApply;
    }

    Need need() const { return need_; }
    int n() const { return n_; }
    int t() const { return t_; }
    const T* x() const { return x_.data(); }  // to apply A to, when need() == kApply
    const T* s() const { return s_.data(); }  // to apply A^H to, when need() == kAdjoint
    T* y() { return y_.data(); }              // receives A x
    T* z() { return z_.data(); }              // receives A^H s

    // Y = A X has been written into y().
    void applied() {
        const int n = n_, t = t_;
        const size_t extent = (size_t)n * t;
        ++k_;
        iterations_ = k_;
        products_ += t;
        int argmax = 0;
        est_ = col_norm(y_.data());
        for (int j = 1; j < t; ++j) {
            double v = col_norm(y_.data() + (size_t)j * n);
            if (v > est_) {
                est_ = v;
                argmax = j;
            }
        }
        if (k_ >= 2 && (est_ > est_old_ || k_ == 2)) best_index_ = current_[argmax];
        if (k_ >= 2 && est_ <= est_old_) {
            est_ = est_old_;
            need_ = kDone;
            return;
        }
        est_old_ = est_;
        if (k_ > itmax_) {
            need_ = kDone;
            return;
        }
        std::swap(s_, s_old_);
        for (size_t i = 0; i < extent; ++i) s_[i] = TE::sign(y_[i]);
        if (TE::kDiscrete && t > 1) {
            bool all = true;
            for (int j = 0; j < t && all; ++j)
                if (!parallel_to_any(s_.data() + (size_t)j * n, s_old_.data(), t)) all = false;
            if (all) {
                need_ = kDone;
                return;
            }
            // MakeColumnsDistinct, :357-370
            for (int j = 0; j < t; ++j)
                for (int attempt = 0; attempt < 8; ++attempt) {
                    if (!parallel_to_any(s_.data() + (size_t)j * n, s_.data(), j) &&
                        !parallel_to_any(s_.data() + (size_t)j * n, s_old_.data(), t))
                        break;
                    fill_signs(s_.data() + (size_t)j * n);
                }
        }
        need_ = kAdjoint;
    }

    // Z = A^H S has been written into z().
    void adjointed() {
        const int n = n_, t = t_;
        products_ += t;
        for (int i = 0; i < n; ++i) {
            double best = 0.0;
            for (int j = 0; j < t; ++j) best = net::max(best, TE::magnitude(z_[(size_t)j * n + i]));
            h_[i] = best;
        }
        if (k_ >= 2 && best_index_ >= 0) {
            double largest = 0.0;
            for (int i = 0; i < n; ++i) largest = net::max(largest, h_[i]);
            if (largest == h_[best_index_]) {
                need_ = kDone;
                return;
            }
        }
        for (int i = 0; i < n; ++i) {
            keys_[i] = -h_[i];
            order_[i] = i;
        }
        net::sort_keys_items(n, keys_.data(), order_.data());
        if (t > 1) {
            bool all_used = true;
            for (int j = 0; j < t; ++j)
                if (!used_[order_[j]]) {
                    all_used = false;
                    break;
                }
            if (all_used) {
                need_ = kDone;
                return;
            }
            // MoveUnusedToFront, :387-402
            int at = 0;
            for (int i = 0; i < n; ++i)
                if (!used_[order_[i]]) scratch_[at++] = order_[i];
            for (int i = 0; i < n; ++i)
                if (used_[order_[i]]) scratch_[at++] = order_[i];
            std::copy(scratch_.begin(), scratch_.end(), order_.begin());
        }
        std::fill(x_.begin(), x_.end(), TE::zero());
        for (int j = 0; j < t; ++j) {
            int index = order_[j];
            current_[j] = index;
            used_[index] = 1;
            x_[(size_t)j * n + index] = TE::one();
        }
        need_ = kApply;
    }

    double value() const { return n_ == 0 ? 0.0 : est_; }
    int iterations() const { return iterations_; }
    int products() const { return products_; }

private:
    void fill_signs(T* p) {
        for (int i = 0; i < n_; ++i) p[i] = rng_.next(2) == 0 ? TE::neg(TE::one()) : TE::one();
    }
    bool is_parallel(const T* u, const T* v) const {
        bool same = true, opposite = true;
        for (int i = 0; i < n_; ++i) {
            if (!TE::eq(u[i], v[i])) same = false;
            if (!TE::eq(u[i], TE::neg(v[i]))) opposite = false;
            if (!same && !opposite) return false;
        }
        return true;
    }
    bool parallel_to_any(const T* col, const T* panel, int count) const {
        for (int j = 0; j < count; ++j)
            if (is_parallel(col, panel + (size_t)j * n_)) return true;
        return false;
    }
    double col_norm(const T* p) const {
        double sum = 0.0;
        for (int i = 0; i < n_; ++i) sum += TE::magnitude(p[i]);
        return sum;
    }

    int n_ = 0, t_ = 1, itmax_ = 2;
    net::Random rng_;
    std::vector<T> x_, y_, s_, s_old_, z_;
    std::vector<double> h_, keys_;
    std::vector<int> order_, scratch_, current_;
    std::vector<char> used_;
    double est_ = 0.0, est_old_ = 0.0;
    int best_index_ = -1, iterations_ = 0, products_ = 0, k_ = 0;
    Need need_ = kDone;
};

}  // namespace tns
