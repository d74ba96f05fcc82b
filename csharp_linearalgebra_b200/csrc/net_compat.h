// Host-side restatements of the .NET runtime behaviour the reference's
// decisions depend on: the seeded System.Random (legacy subtractive
// generator), Array.Sort(double[], int[]) (NaN prepass + introsort), and
// System.Numerics.Complex arithmetic. normest1 draws its probe signs from
// the former (src/Tensile/NormEstimate.cs:163,301-305) and orders its
// candidates with the latter (:372-381); both shape the estimate, and through
// it expm's degree and scaling.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <utility>

namespace tns {
namespace net {

class Random {
public:
    explicit Random(int seed) {
        const int mbig = 2147483647, mseed = 161803398;
        int subtraction = seed == std::numeric_limits<int>::min() ? mbig : std::abs(seed);
        int mj = mseed - subtraction;
        a_[55] = mj;
        int mk = 1;
        for (int i = 1; i < 55; ++i) {
            int ii = (21 * i) % 55;
            a_[ii] = mk;
            mk = mj - mk;
            if (mk < 0) mk += mbig;
            mj = a_[ii];
        }
        for (int k = 1; k < 5; ++k)
            for (int i = 1; i < 56; ++i) {
                a_[i] -= a_[1 + (i + 30) % 55];
                if (a_[i] < 0) a_[i] += mbig;
            }
        a_[0] = 0;
    }
    // Random.Next(maxValue)
    int next(int max_value) { return (int)(sample() * max_value); }
    // Random.NextDouble()
    double sample() { return internal() * (1.0 / 2147483647); }

private:
    int internal() {
        if (++next_ >= 56) next_ = 1;
        if (++nextp_ >= 56) nextp_ = 1;
        int r = a_[next_] - a_[nextp_];
        if (r == 2147483647) --r;
        if (r < 0) r += 2147483647;
        a_[next_] = r;
        return r;
    }
    int a_[56];
    int next_ = 0, nextp_ = 21;
};

// Array.Sort(keys, items) with the default comparer.
inline void sort_keys_items(int n, double* k, int* v) {
    struct S {
        double* k;
        int* v;
        void sw(int i, int j) {
            std::swap(k[i], k[j]);
            std::swap(v[i], v[j]);
        }
        void sig(int i, int j) {
            if (k[i] > k[j]) sw(i, j);
        }
        void ins(int lo, int len) {
            for (int i = 0; i < len - 1; ++i) {
                double t = k[lo + i + 1];
                int tv = v[lo + i + 1];
                int j = i;
                while (j >= 0 && t < k[lo + j]) {
                    k[lo + j + 1] = k[lo + j];
                    v[lo + j + 1] = v[lo + j];
                    --j;
                }
                k[lo + j + 1] = t;
                v[lo + j + 1] = tv;
            }
        }
        void down(int lo, int i, int n) {
            double d = k[lo + i - 1];
            int dv = v[lo + i - 1];
            while (i <= (n >> 1)) {
                int c = 2 * i;
                if (c < n && k[lo + c - 1] < k[lo + c]) ++c;
                if (!(d < k[lo + c - 1])) break;
                k[lo + i - 1] = k[lo + c - 1];
                v[lo + i - 1] = v[lo + c - 1];
                i = c;
            }
            k[lo + i - 1] = d;
            v[lo + i - 1] = dv;
        }
        void heap(int lo, int n) {
            for (int i = n >> 1; i >= 1; --i) down(lo, i, n);
            for (int i = n; i > 1; --i) {
                sw(lo, lo + i - 1);
                down(lo, 1, i - 1);
            }
        }
        int part(int lo, int len) {
            int hi = len - 1, mid = hi >> 1;
            sig(lo, lo + mid);
            sig(lo, lo + hi);
            sig(lo + mid, lo + hi);
            double pivot = k[lo + mid];
            sw(lo + mid, lo + hi - 1);
            int l = 0, r = hi - 1;
            while (l < r) {
                while (pivot > k[lo + (++l)]) {
                }
                while (pivot < k[lo + (--r)]) {
                }
                if (l >= r) break;
                sw(lo + l, lo + r);
            }
            if (l != hi - 1) sw(lo + l, lo + hi - 1);
            return l;
        }
        void intro(int lo, int len, int depth) {
            while (len > 1) {
                if (len <= 16) {
                    if (len == 2) {
                        sig(lo, lo + 1);
                        return;
                    }
                    if (len == 3) {
                        sig(lo, lo + 1);
                        sig(lo, lo + 2);
                        sig(lo + 1, lo + 2);
                        return;
                    }
                    ins(lo, len);
                    return;
                }
                if (depth == 0) {
                    heap(lo, len);
                    return;
                }
                --depth;
                int p = part(lo, len);
                intro(lo + p + 1, len - (p + 1), depth);
                len = p;
            }
        }
    };
    if (n <= 1) return;
    int left = 0;
    for (int i = 0; i < n; ++i)
        if (std::isnan(k[i])) {
            std::swap(k[left], k[i]);
            std::swap(v[left], v[i]);
            ++left;
        }
    if (left == n) return;
    int len = n - left;
    int lg = 0;
    for (unsigned x = (unsigned)len; x >>= 1;) ++lg;
    S{k + left, v + left}.intro(0, len, 2 * (lg + 1));
}

inline double max(double a, double b) {
    if (a != b) {
        if (!std::isnan(a)) return b < a ? a : b;
        return a;
    }
    return std::signbit(b) ? a : b;
}
inline double min(double a, double b) {
    if (a != b) {
        if (!std::isnan(a)) return a < b ? a : b;
        return a;
    }
    return std::signbit(a) ? a : b;
}

struct Cx {
    double re = 0.0, im = 0.0;
};
inline bool operator==(Cx a, Cx b) { return a.re == b.re && a.im == b.im; }
inline Cx operator-(Cx a) { return {-a.re, -a.im}; }
inline Cx mul(Cx a, Cx b) { return {(a.re * b.re) - (a.im * b.im), (a.im * b.re) + (a.re * b.im)}; }
inline Cx div(Cx l, Cx r) {
    double a = l.re, b = l.im, c = r.re, d = r.im;
    if (std::fabs(d) < std::fabs(c)) {
        double doc = d / c;
        return {(a + b * doc) / (c + d * doc), (b - a * doc) / (c + d * doc)};
    }
    double cod = c / d;
    return {(b + a * cod) / (d + c * cod), (-a + b * cod) / (d + c * cod)};
}
inline double abs(Cx z) {
    double a = std::fabs(z.re), b = std::fabs(z.im);
    double small = a < b ? a : b, large = a < b ? b : a;
    if (small == 0.0) return large;
    if (std::isinf(large) && !std::isnan(small)) return std::numeric_limits<double>::infinity();
    double ratio = small / large;
    return large * std::sqrt(1.0 + ratio * ratio);
}
inline Cx exp(Cx z) {
    double e = std::exp(z.re);
    return {e * std::cos(z.im), e * std::sin(z.im)};
}

}  // namespace net
}  // namespace tns
