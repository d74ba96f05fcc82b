// exp(tA)B by Al-Mohy & Higham 2011 truncated Taylor (the reference's
// MatrixExponentialAction.Dense + Run, src/Tensile/MatrixExponentialAction.cs:149-178,
// 239-320), for one matrix or a batch of independent ones.
//
// The parameter selection runs on the host in the reference's order (trace
// shift, ||A - mu I||_1, the sharp ||A^p||^(1/p) bounds from normest1 with
// every estimator of the batch advanced together, the (m, s) search). The
// whole Taylor recurrence -- every operator application, the scaling of the
// new term, its accumulation into F, both infinity norms and the early-exit
// test -- then runs in ONE cooperative launch: taylor_kernel.
//
// taylor_kernel. Each matrix is worked on by a group of CTAs ("lanes"); the
// rows of A, F and the work panels are split among them. One application of
// A to the n x c work panel X is, per CTA, the product of its rows of A with
// all of X, staged through shared memory by cp.async in 32-deep k tiles (a
// 4-stage ring); one thread owns one (row, column) pair and sums in k order
// with the reference's rounding (PanelProduct.Apply's axpy order, a product
// and a sum per term; the complex operator's four real sums then
// (pr - qi, pi + qr), LinearOperators.cs:262-282). The reference skips a term
// whose x is zero; forming it instead adds +-0 to a sum that is never -0,
// which changes nothing as long as A is finite, so the skip is kept (as a
// compare and a select) only in launches with a non-finite operator. The epilogue scales
// the sums by t/(s(j+1)) into the next work panel, adds them into F and forms
// both row sums of moduli in column order (InfinityNorm). Every CTA writes
// its largest row sums to its slot, the group meets at a barrier, and every
// CTA folds the slots to the same two norms and takes the same exit
// decision: c1 + c2 <= u ||F||_inf ends the inner loop on the device, with no
// host round trip. The panels alternate between two buffers, so no CTA
// overwrites a panel another is still reading.
//
// Groups and the barrier. A host-side list schedule gives each matrix a width
// (CTAs) from its share of the batch's work and places it, longest first, on
// the lanes that free up earliest; each CTA then works through its list of
// (matrix, rank) in the order of the schedule's start times, which is one
// total order for every lane, so no group can wait on a lane that waits on
// it. A group of one CTA synchronises with __syncthreads; a wider group on a
// counter in global memory (release/acquire), with a bounded spin: a wait
// gives up after 2 s in which no barrier anywhere in the launch advanced,
// records a device error and returns, and the host reports TNS_E_TIMEOUT.

#include "batch.cuh"
#include "device_util.cuh"
#include "net_compat.h"
#include "tns_internal.h"

#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

namespace tns {

namespace {

constexpr int kThreadsT = 512;  // threads per CTA: (row, column slot) pairs

// The thread layout and the inner loop's form, per launch: SLOTS column slots
// per row (8 for panels of up to 8 columns, else 16), CPT columns per slot
// (c + SLOTS q), ROWS = 512 / SLOTS rows per chunk of a CTA's row range.
// SKIP keeps the reference's skip of a zero x term explicitly (a compare and
// a select per term). Without it the term is always formed: that adds +-0 to
// a sum that is never -0, the same bits whenever A is finite; the host takes
// that form only when every ||A - mu I||_1 of the launch is finite (0 * inf
// would otherwise differ from a skip).
template <int SLOTS_, int CPT_, bool SKIP_>
struct Shape {
    static constexpr int SLOTS = SLOTS_, CPT = CPT_, ROWS = kThreadsT / SLOTS_;
    static constexpr bool SKIP = SKIP_;
};
constexpr int kKT = 32;                    // k per staged tile
constexpr int kStagesT = 4;                // cp.async ring depth
constexpr double kU = 1.1102230246251565e-16;
constexpr int kDevTimeoutGroup = 4;  // DeviceError: a group barrier of the Taylor kernel gave up

struct TaylorDesc {
    const double* a;   // the shifted matrix A - mu I, ld lda
    const double* b;   // B, ld ldb
    double* f;         // the result F, ld ldp
    double* w0;        // work panels, ld ldp
    double* w1;
    const double* coeff;        // m coefficients t / (s (j + 1))
    double* partials;           // [2][width][2]
    unsigned long long* bar;    // the group's barrier counter (zero at launch)
    int* out;                   // [applications, early exits]
    int n, lda, ldb, ldp;
    int m, s, width, rows_per;  // rows_per: rows per CTA, a multiple of 8
    double eta_re, eta_im;
    int eta_one;
};

struct TaylorPlan {
    int matrix, rank;
};

struct TaylorLaunch {
    const TaylorDesc* descs;
    const TaylorPlan* plan;
    const int* plan_off;  // gridDim.x + 1 offsets into plan
    int ncols;
    int* err;
    unsigned long long* progress;  // every barrier arrival in the launch
};

__device__ __forceinline__ void cp16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// The group's barrier number `target / width`. False when it gave up (the
// error flag is then set); every thread of the CTA gets the same answer.
__device__ bool group_sync(const TaylorDesc& d, unsigned long long target, const TaylorLaunch& L, int* s_flag) {
    __syncthreads();
    if (d.width == 1) return true;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(d.bar, 1ull);
        atomicAdd(L.progress, 1ull);
        int ok = 1;
        if (ld_acquire(d.bar) < target) {
            unsigned long long start = global_timer_ns();
            unsigned long long beat = ld_acquire(L.progress);
            for (unsigned it = 1;; ++it) {
                if (ld_acquire(d.bar) >= target) break;
                if (it > 64) __nanosleep(64);
                if ((it & 127u) == 0) {
                    if (*reinterpret_cast<volatile int*>(L.err) != 0) {
                        ok = 0;
                        break;
                    }
                    const unsigned long long now = global_timer_ns();
                    const unsigned long long b2 = ld_acquire(L.progress);
                    if (b2 != beat) {
                        beat = b2;
                        start = now;
                    } else if (now - start > kWaitTimeoutNs) {
                        atomicCAS(L.err, 0, kDevTimeoutGroup);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        __threadfence();
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

// Largest of non-negative values with Math.Max's NaN rule (any NaN wins).
struct NormAcc {
    double v = 0.0;
    bool nan = false;
    __device__ void add(double x) {
        if (isnan(x)) nan = true;
        else if (x > v) v = x;
    }
    __device__ double value() const { return nan ? __longlong_as_double(0x7ff8000000000000ll) : v; }
};

// Fold the CTA's two norm accumulators (every thread holds its own) into
// s_part[0..1] (thread 0's view after the sync).
__device__ void cta_fold(NormAcc a0, NormAcc a1, double* s_red, int* s_nan, double* s_part) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double x0 = __shfl_xor_sync(0xffffffffu, a0.v, o), x1 = __shfl_xor_sync(0xffffffffu, a1.v, o);
        int n0 = __shfl_xor_sync(0xffffffffu, (int)a0.nan, o), n1 = __shfl_xor_sync(0xffffffffu, (int)a1.nan, o);
        a0.v = x0 > a0.v ? x0 : a0.v;
        a1.v = x1 > a1.v ? x1 : a1.v;
        a0.nan = a0.nan || n0;
        a1.nan = a1.nan || n1;
    }
    if (lane == 0) {
        s_red[warp] = a0.v;
        s_red[32 + warp] = a1.v;
        s_nan[warp] = a0.nan;
        s_nan[32 + warp] = a1.nan;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        NormAcc r0, r1;
        for (int w = 0; w < kThreadsT / 32; ++w) {
            r0.v = s_red[w] > r0.v ? s_red[w] : r0.v;
            r1.v = s_red[32 + w] > r1.v ? s_red[32 + w] : r1.v;
            r0.nan = r0.nan || s_nan[w];
            r1.nan = r1.nan || s_nan[32 + w];
        }
        s_part[0] = r0.value();
        s_part[1] = r1.value();
    }
}

// Publish the CTA's two values, meet the group, and leave the group's two
// norms in s_norm (every thread). False if the barrier gave up.
__device__ bool group_norms(const TaylorDesc& d, int rank, unsigned long long& phase, const TaylorLaunch& L,
                            NormAcc a0, NormAcc a1, double* s_red, int* s_nan, double* s_part, double* s_norm,
                            int* s_flag) {
    cta_fold(a0, a1, s_red, s_nan, s_part);
    const int parity = (int)(phase & 1);
    if (d.width > 1 && threadIdx.x == 0) {
        double* slot = d.partials + ((size_t)parity * d.width + rank) * 2;
        slot[0] = s_part[0];
        slot[1] = s_part[1];
    }
    ++phase;
    if (!group_sync(d, phase * (unsigned long long)d.width, L, s_flag)) return false;
    if (d.width == 1) {
        if (threadIdx.x == 0) {
            s_norm[0] = s_part[0];
            s_norm[1] = s_part[1];
        }
    } else if (threadIdx.x < 32) {
        NormAcc r0, r1;
        for (int r = threadIdx.x; r < d.width; r += 32) {
            const double* slot = d.partials + ((size_t)parity * d.width + r) * 2;
            r0.add(__ldcg(slot));
            r1.add(__ldcg(slot + 1));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double x0 = __shfl_xor_sync(0xffffffffu, r0.v, o), x1 = __shfl_xor_sync(0xffffffffu, r1.v, o);
            int n0 = __shfl_xor_sync(0xffffffffu, (int)r0.nan, o), n1 = __shfl_xor_sync(0xffffffffu, (int)r1.nan, o);
            r0.v = x0 > r0.v ? x0 : r0.v;
            r1.v = x1 > r1.v ? x1 : r1.v;
            r0.nan = r0.nan || n0;
            r1.nan = r1.nan || n1;
        }
        if (threadIdx.x == 0) {
            s_norm[0] = r0.value();
            s_norm[1] = r1.value();
        }
    }
    __syncthreads();
    return true;
}

template <bool CPLX>
__device__ __forceinline__ double modulus(double re, double im) {
    if constexpr (CPLX) return cabs_net(re, im);
    else return fabs(re);
}

// Row sums of moduli over the columns in column order (InfinityNorm,
// ComplexKernels.cs:164-180 / Norms.cs:50-66): the 8 lanes of a row hold its
// columns c + SLOTS q; every lane ends with its row's sum.
template <class S>
__device__ __forceinline__ double row_sum(const double (&v)[S::CPT], int ncols) {
    const int base = threadIdx.x & (32 - S::SLOTS);  // first lane of this row in the warp
    double sum = 0.0;
#pragma unroll
    for (int q = 0; q < S::CPT; ++q)
#pragma unroll
        for (int c = 0; c < S::SLOTS; ++c) {
            const double x = __shfl_sync(0xffffffffu, v[q], base + c);
            if (q * S::SLOTS + c < ncols) sum = add_rn(sum, x);
        }
    return sum;
}

template <bool CPLX, class S>
struct Tiles {
    static constexpr int ES = CPLX ? 2 : 1;                 // doubles per element
    static constexpr int XS = CPLX ? kKT + 1 : kKT + 2;     // elements per staged X column
    static constexpr int A_DOUBLES = kKT * S::ROWS * ES;
    static constexpr int X_DOUBLES = S::SLOTS * S::CPT * XS * ES;
    static constexpr int STAGE = A_DOUBLES + X_DOUBLES;
    static constexpr size_t SMEM = sizeof(double) * (size_t)STAGE * kStagesT;
};

// Stage k tile [k0, k0 + kKT) of the CTA's rows [r0, r0 + rows) of A and of
// the work panel x (all columns) into stage buffer `buf`.
template <bool CPLX, class S>
__device__ __forceinline__ void stage_tile(double* buf, const TaylorDesc& d, const double* x, int ncols, int r0,
                                           int rows, int k0) {
    using T = Tiles<CPLX, S>;
    constexpr int R = S::ROWS;
    double* sA = buf;
    double* sX = buf + T::A_DOUBLES;
    const int tid = threadIdx.x;
    if constexpr (CPLX) {
        for (int e = tid; e < kKT * R; e += kThreadsT) {
            const int k = e / R, r = e % R;
            if (r < rows) cp16(sA + (k * R + r) * 2, d.a + ((size_t)(k0 + k) * d.lda + r0 + r) * 2);
        }
        for (int e = tid; e < ncols * kKT; e += kThreadsT) {
            const int col = e / kKT, k = e % kKT;
            cp16(sX + (col * T::XS + k) * 2, x + ((size_t)col * d.ldp + k0 + k) * 2);
        }
    } else {
        for (int e = tid; e < kKT * (R / 2); e += kThreadsT) {
            const int k = e / (R / 2), rp = (e % (R / 2)) * 2;
            if (rp < rows) cp16(sA + k * R + rp, d.a + (size_t)(k0 + k) * d.lda + r0 + rp);
        }
        for (int e = tid; e < ncols * (kKT / 2); e += kThreadsT) {
            const int col = e / (kKT / 2), kp = (e % (kKT / 2)) * 2;
            cp16(sX + col * T::XS + kp, x + (size_t)col * d.ldp + k0 + kp);
        }
    }
}

// acc := (rows r0.. of A) * x for this thread's (row, columns), in k order.
template <bool CPLX, class S>
__device__ __forceinline__ void product_chunk(double* smem, const TaylorDesc& d, const double* x, int ncols, int r0,
                                              int rows, double (&acc)[S::CPT][CPLX ? 4 : 1]) {
    using T = Tiles<CPLX, S>;
    constexpr int R = S::ROWS;
    const int rr = threadIdx.x / S::SLOTS, c = threadIdx.x % S::SLOTS;
#pragma unroll
    for (int q = 0; q < S::CPT; ++q)
#pragma unroll
        for (int z = 0; z < (CPLX ? 4 : 1); ++z) acc[q][z] = 0.0;
    const int n = d.n;
    const int ktiles = (n + kKT - 1) / kKT;
#pragma unroll
    for (int st = 0; st < kStagesT - 1; ++st) {
        if (st < ktiles) stage_tile<CPLX, S>(smem + st * T::STAGE, d, x, ncols, r0, rows, st * kKT);
        cp_commit();
    }
    bool col_ok[S::CPT];
#pragma unroll
    for (int q = 0; q < S::CPT; ++q) col_ok[q] = c + q * S::SLOTS < ncols;
    for (int kt = 0; kt < ktiles; ++kt) {
        cp_wait<kStagesT - 2>();
        __syncthreads();
        const int nxt = kt + kStagesT - 1;
        if (nxt < ktiles) stage_tile<CPLX, S>(smem + (nxt % kStagesT) * T::STAGE, d, x, ncols, r0, rows, nxt * kKT);
        cp_commit();
        const double* sA = smem + (kt % kStagesT) * T::STAGE;
        const double* sX = sA + T::A_DOUBLES;
        const int klen = min(kKT, n - kt * kKT);
        if (rr < rows) {
            if constexpr (CPLX) {
                const double2* a2 = reinterpret_cast<const double2*>(sA) + rr;
                const double2* x2 = reinterpret_cast<const double2*>(sX) + c * T::XS;
#pragma unroll 4
                for (int kk = 0; kk < klen; ++kk) {
                    const double2 av = a2[kk * R];
#pragma unroll
                    for (int q = 0; q < S::CPT; ++q) {
                        if (!col_ok[q]) continue;
                        const double2 xv = x2[q * S::SLOTS * T::XS + kk];
                        if constexpr (S::SKIP) {
                            const bool nr = xv.x != 0.0, ni = xv.y != 0.0;
                            acc[q][0] = add_rn(acc[q][0], nr ? mul_rn(xv.x, av.x) : 0.0);  // pr
                            acc[q][2] = add_rn(acc[q][2], nr ? mul_rn(xv.x, av.y) : 0.0);  // qr
                            acc[q][1] = add_rn(acc[q][1], ni ? mul_rn(xv.y, av.x) : 0.0);  // pi
                            acc[q][3] = add_rn(acc[q][3], ni ? mul_rn(xv.y, av.y) : 0.0);  // qi
                        } else {
                            acc[q][0] = add_rn(acc[q][0], mul_rn(xv.x, av.x));
                            acc[q][2] = add_rn(acc[q][2], mul_rn(xv.x, av.y));
                            acc[q][1] = add_rn(acc[q][1], mul_rn(xv.y, av.x));
                            acc[q][3] = add_rn(acc[q][3], mul_rn(xv.y, av.y));
                        }
                    }
                }
            } else {
                const double* a1 = sA + rr;
                const double* x1 = sX + c * T::XS;
#pragma unroll 4
                for (int kk = 0; kk < klen; ++kk) {
                    const double av = a1[kk * R];
#pragma unroll
                    for (int q = 0; q < S::CPT; ++q) {
                        if (!col_ok[q]) continue;
                        const double xv = x1[q * S::SLOTS * T::XS + kk];
                        if constexpr (S::SKIP) acc[q][0] = add_rn(acc[q][0], xv != 0.0 ? mul_rn(xv, av) : 0.0);
                        else acc[q][0] = add_rn(acc[q][0], mul_rn(xv, av));
                    }
                }
            }
        }
    }
    cp_wait<0>();
    __syncthreads();
}

template <bool CPLX, class S>
__global__ void __launch_bounds__(kThreadsT, 1) taylor_kernel(const __grid_constant__ TaylorLaunch L) {
    constexpr int CPT = S::CPT, R = S::ROWS;
    extern __shared__ __align__(128) double smem[];
    __shared__ double s_red[64];
    __shared__ int s_nan[64];
    __shared__ double s_part[2];
    __shared__ double s_norm[2];
    __shared__ int s_flag;
    const int ncols = L.ncols;
    const int rr = threadIdx.x / S::SLOTS, cs = threadIdx.x % S::SLOTS;
    for (int e = L.plan_off[blockIdx.x]; e < L.plan_off[blockIdx.x + 1]; ++e) {
        const TaylorPlan pl = L.plan[e];
        const TaylorDesc d = L.descs[pl.matrix];
        const int rank = pl.rank;
        const int rbeg = rank * d.rows_per, rend = min(d.n, rbeg + d.rows_per);
        unsigned long long phase = 0;
        const size_t es = CPLX ? 2 : 1;

        // F := B, work := B, c1 = ||B||_inf (Run, :274-276, :285).
        NormAcc n0, n1;
        for (int r0 = rbeg; r0 < rend; r0 += R) {
            const int i = r0 + rr;
            const bool row_ok = i < rend;
            double v[CPT];
#pragma unroll
            for (int q = 0; q < CPT; ++q) {
                const int col = cs + q * S::SLOTS;
                v[q] = 0.0;
                if (row_ok && col < ncols) {
                    const size_t bi = ((size_t)col * d.ldb + i) * es, pi = ((size_t)col * d.ldp + i) * es;
                    const double re = d.b[bi], im = CPLX ? d.b[bi + 1] : 0.0;
                    d.f[pi] = re;
                    d.w0[pi] = re;
                    if (CPLX) {
                        d.f[pi + 1] = im;
                        d.w0[pi + 1] = im;
                    }
                    v[q] = modulus<CPLX>(re, im);
                }
            }
            const double rs = row_sum<S>(v, ncols);
            if (row_ok) n0.add(rs);
        }
        if (!group_norms(d, rank, phase, L, n0, n1, s_red, s_nan, s_part, s_norm, &s_flag)) return;
        double c1 = s_norm[0];

        int applications = 0, early = 0;
        double* win = d.w0;
        double* wout = d.w1;
        for (int step = 0; step < d.s; ++step) {
            for (int j = 0; j < d.m; ++j) {
                const double coeff = d.coeff[j];
                NormAcc nw, nf;
                for (int r0 = rbeg; r0 < rend; r0 += R) {
                    const int rows = min(R, rend - r0);
                    double acc[CPT][CPLX ? 4 : 1];
                    product_chunk<CPLX, S>(smem, d, win, ncols, r0, rows, acc);
                    const int i = r0 + rr;
                    const bool row_ok = rr < rows;
                    double vw[CPT], vf[CPT];
#pragma unroll
                    for (int q = 0; q < CPT; ++q) {
                        const int col = cs + q * S::SLOTS;
                        vw[q] = 0.0;
                        vf[q] = 0.0;
                        if (row_ok && col < ncols) {
                            const size_t pi = ((size_t)col * d.ldp + i) * es;
                            if constexpr (CPLX) {
                                // next = A work; work := Scale(next, coefficient) (ScaleInto, :441-452)
                                const double yr = sub_rn(acc[q][0], acc[q][3]), yi = add_rn(acc[q][1], acc[q][2]);
                                const double wr = mul_rn(yr, coeff), wi = mul_rn(yi, coeff);
                                wout[pi] = wr;
                                wout[pi + 1] = wi;
                                // F += work (AddInto, :466-476)
                                const double fr = add_rn(d.f[pi], wr), fi = add_rn(d.f[pi + 1], wi);
                                d.f[pi] = fr;
                                d.f[pi + 1] = fi;
                                vw[q] = cabs_net(wr, wi);
                                vf[q] = cabs_net(fr, fi);
                            } else {
                                const double w = mul_rn(acc[q][0], coeff);
                                wout[pi] = w;
                                const double fv = add_rn(d.f[pi], w);
                                d.f[pi] = fv;
                                vw[q] = fabs(w);
                                vf[q] = fabs(fv);
                            }
                        }
                    }
                    const double sw = row_sum<S>(vw, ncols), sf = row_sum<S>(vf, ncols);
                    if (row_ok) {
                        nw.add(sw);
                        nf.add(sf);
                    }
                }
                if (!group_norms(d, rank, phase, L, nw, nf, s_red, s_nan, s_part, s_norm, &s_flag)) return;
                const double c2 = s_norm[0], fnorm = s_norm[1];
                ++applications;
                double* tmp = win;
                win = wout;
                wout = tmp;
                // The remaining terms cannot move F at this precision (:298-305).
                if (add_rn(c1, c2) <= mul_rn(kU, fnorm)) {
                    ++early;
                    break;
                }
                c1 = c2;
            }
            // F *= eta (ScaleInPlace, :455-464); work := F (CopyInto); c1 = ||work||_inf.
            NormAcc ne, unused;
            for (int r0 = rbeg; r0 < rend; r0 += R) {
                const int i = r0 + rr;
                const bool row_ok = i < rend;
                double v[CPT];
#pragma unroll
                for (int q = 0; q < CPT; ++q) {
                    const int col = cs + q * S::SLOTS;
                    v[q] = 0.0;
                    if (row_ok && col < ncols) {
                        const size_t pi = ((size_t)col * d.ldp + i) * es;
                        double re = d.f[pi], im = CPLX ? d.f[pi + 1] : 0.0;
                        if (!d.eta_one) {
                            if constexpr (CPLX) {
                                // Complex multiply (left = F, right = eta), .NET's order of terms.
                                const double nr = sub_rn(mul_rn(re, d.eta_re), mul_rn(im, d.eta_im));
                                const double ni = add_rn(mul_rn(im, d.eta_re), mul_rn(re, d.eta_im));
                                re = nr;
                                im = ni;
                            } else {
                                re = mul_rn(re, d.eta_re);
                            }
                            d.f[pi] = re;
                            if (CPLX) d.f[pi + 1] = im;
                        }
                        win[pi] = re;
                        if (CPLX) win[pi + 1] = im;
                        v[q] = modulus<CPLX>(re, im);
                    }
                }
                const double rs = row_sum<S>(v, ncols);
                if (row_ok) ne.add(rs);
            }
            if (!group_norms(d, rank, phase, L, ne, unused, s_red, s_nan, s_part, s_norm, &s_flag)) return;
            c1 = s_norm[0];
        }
        if (rank == 0 && threadIdx.x == 0) {
            d.out[0] = applications;
            d.out[1] = early;
        }
    }
}

// ---- host ----------------------------------------------------------------

__global__ void trace_batch_kernel(const __grid_constant__ Batch<SumDesc> b, bool cplx) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= b.count) return;
    const SumDesc& d = batch_item(b, k);
    double re = 0.0, im = 0.0;
    for (int i = 0; i < d.m; ++i) {
        if (!cplx) {
            re = add_rn(re, d.a[(size_t)i * d.ld + i]);
        } else {
            const double2 z = reinterpret_cast<const double2*>(d.a)[(size_t)i * d.ld + i];
            re = add_rn(re, z.x);
            im = add_rn(im, z.y);
        }
    }
    d.out[0] = re;
    d.out[1] = im;
}

// The trace of every matrix (Trace, :418-423; complex per part), to the host.
std::vector<double> traces(Context& ctx, const std::vector<const DMat*>& as) {
    const size_t cnt = as.size();
    DBuf out(ctx, sizeof(double) * 2 * cnt);
    std::vector<SumDesc> v;
    for (size_t k = 0; k < cnt; ++k) v.push_back(SumDesc{as[k]->p, as[k]->rows, as[k]->rows, as[k]->ld(), out.as<double>() + 2 * k});
    Batch<SumDesc> b = make_batch(ctx, v);
    trace_batch_kernel<<<(int)((cnt + 127) / 128), 128, 0, ctx.stream>>>(b, as[0]->cplx);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
    std::vector<double> h(2 * cnt);
    TNS_CUDA(cudaMemcpyAsync(h.data(), out.p, sizeof(double) * 2 * cnt, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    return h;
}

const int kEll = 2, kMaxPower = 8;

template <bool CPLX, class S>
void launch_taylor(Context& ctx, const TaylorLaunch& L, int grid) {
    using T = Tiles<CPLX, S>;
    TNS_CUDA(cudaFuncSetAttribute(taylor_kernel<CPLX, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM));
    void* args[] = {const_cast<TaylorLaunch*>(&L)};
    TNS_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(taylor_kernel<CPLX, S>), dim3(grid),
                                         dim3(kThreadsT), args, T::SMEM, ctx.stream));
    ctx.kernel_launches++;
}

template <bool CPLX, class S>
int resident_ctas(Context& ctx) {
    using T = Tiles<CPLX, S>;
    TNS_CUDA(cudaFuncSetAttribute(taylor_kernel<CPLX, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM));
    int per_sm = 0;
    TNS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, taylor_kernel<CPLX, S>, kThreadsT, T::SMEM));
    if (per_sm < 1) fail(TNS_E_DEVICE, "the Taylor kernel cannot be resident on this device");
    return per_sm * ctx.num_sms;
}

// One kernel instance per (element type, layout, skip form); L null: only the
// count of resident CTAs.
template <bool CPLX, bool SKIP>
int taylor_dispatch(Context& ctx, int layout, const TaylorLaunch* L, int grid) {
    using S8 = Shape<8, 1, SKIP>;
    using S16 = Shape<16, 1, SKIP>;
    using S16x2 = Shape<16, 2, SKIP>;
    if (!L) return layout == 0 ? resident_ctas<CPLX, S8>(ctx) : layout == 1 ? resident_ctas<CPLX, S16>(ctx)
                                                                              : resident_ctas<CPLX, S16x2>(ctx);
    if (layout == 0) launch_taylor<CPLX, S8>(ctx, *L, grid);
    else if (layout == 1) launch_taylor<CPLX, S16>(ctx, *L, grid);
    else launch_taylor<CPLX, S16x2>(ctx, *L, grid);
    return grid;
}

int taylor(Context& ctx, bool cplx, bool skip, int layout, const TaylorLaunch* L, int grid) {
    if (cplx) return skip ? taylor_dispatch<true, true>(ctx, layout, L, grid) : taylor_dispatch<true, false>(ctx, layout, L, grid);
    return skip ? taylor_dispatch<false, true>(ctx, layout, L, grid) : taylor_dispatch<false, false>(ctx, layout, L, grid);
}

// The list schedule: each matrix's width from its share of the work, then,
// longest first, onto the lanes that free up earliest. Returns per-lane lists
// of (matrix, rank) sorted by (start time, placement order).
struct Sched {
    std::vector<int> width, rows_per;
    std::vector<int> offsets;
    std::vector<TaylorPlan> plan;
};

Sched schedule(const std::vector<int>& n, const std::vector<double>& apps, int ncols, int lanes, int chunk_rows) {
    const size_t cnt = n.size();
    Sched sc;
    sc.width.assign(cnt, 1);
    sc.rows_per.assign(cnt, 8);
    // Time model per application: n x (rows per CTA) x ncols element steps
    // at `rate` per CTA, plus a barrier overhead for groups wider than one.
    // (Measured on the sweep: widths in proportion to the work share beat
    // rounding the rows per CTA up to whole chunks.)
    const double rate = 1.0e10, bar_wide = 2.0e-6, bar_one = 0.5e-6;
    (void)chunk_rows;
    std::vector<double> work(cnt);
    double total = 0.0;
    for (size_t k = 0; k < cnt; ++k) {
        work[k] = apps[k] * (double)n[k] * n[k] * ncols;
        total += work[k];
    }
    std::vector<double> dur(cnt);
    for (size_t k = 0; k < cnt; ++k) {
        const int max_w = std::max(1, std::min(lanes, (n[k] + 7) / 8));
        int w = total > 0.0 ? (int)std::lround(lanes * work[k] / total) : 1;
        w = std::clamp(w, 1, max_w);
        int rp = round_up((n[k] + w - 1) / w, 8);
        w = (n[k] + rp - 1) / rp;  // no rank without rows
        sc.width[k] = w;
        sc.rows_per[k] = rp;
        dur[k] = apps[k] * ((double)n[k] * rp * ncols / rate + (w > 1 ? bar_wide : bar_one));
    }
    std::vector<int> order(cnt);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return dur[x] > dur[y]; });
    std::vector<double> free_at(lanes, 0.0);
    struct Entry {
        double start;
        int seq, matrix, rank;
    };
    std::vector<std::vector<Entry>> per_lane(lanes);
    std::vector<int> idx(lanes);
    int seq = 0;
    for (int k : order) {
        const int w = sc.width[k];
        std::iota(idx.begin(), idx.end(), 0);
        std::partial_sort(idx.begin(), idx.begin() + w, idx.end(),
                          [&](int x, int y) { return free_at[x] < free_at[y] || (free_at[x] == free_at[y] && x < y); });
        double start = 0.0;
        for (int r = 0; r < w; ++r) start = std::max(start, free_at[idx[r]]);
        for (int r = 0; r < w; ++r) {
            per_lane[idx[r]].push_back(Entry{start, seq, k, r});
            free_at[idx[r]] = start + dur[k];
        }
        ++seq;
    }
    sc.offsets.assign(lanes + 1, 0);
    for (int l = 0; l < lanes; ++l) {
        auto& v = per_lane[l];
        std::sort(v.begin(), v.end(), [](const Entry& x, const Entry& y) { return x.start < y.start || (x.start == y.start && x.seq < y.seq); });
        sc.offsets[l + 1] = sc.offsets[l] + (int)v.size();
        for (auto& e : v) sc.plan.push_back(TaylorPlan{e.matrix, e.rank});
    }
    return sc;
}

}  // namespace

void expmv_batch(Context& ctx, const std::vector<const DMat*>& as, const std::vector<const DMat*>& bs, double t,
                 std::vector<DMat>& results, std::vector<ExpmvInfo>& infos, int select_only_cols) {
    const size_t cnt = as.size();
    results.clear();
    results.resize(cnt);
    infos.assign(cnt, ExpmvInfo{});
    if (cnt == 0) return;
    const bool cplx = as[0]->cplx;
    const bool select_only = select_only_cols > 0;
    const int ncols = select_only ? select_only_cols : bs[0]->cols;
    for (size_t k = 0; k < cnt; ++k)
        if (as[k]->cplx != cplx || as[k]->rows < 1 ||
            (!select_only && (bs[k]->cols != ncols || bs[k]->rows != as[k]->rows)))
            fail(TNS_E_ARGUMENT, "internal: an exponential-action batch mixes element types or panel widths");

    // mu = trace / n (per part for complex), A - mu I, ||A - mu I||_1
    // (Expmv, :131-141; complex MatrixExponentialAction.Complex.cs:57-61; Dense, :157).
    std::vector<double> tr = traces(ctx, as);
    std::vector<DMat> sh(cnt);
    std::vector<double> mu_re(cnt), mu_im(cnt, 0.0);
    std::vector<const DMat*> shp(cnt);
    for (size_t k = 0; k < cnt; ++k) {
        const int n = as[k]->rows;
        mu_re[k] = tr[2 * k] / n;
        if (cplx) mu_im[k] = tr[2 * k + 1] / n;
        sh[k] = DMat(ctx, n, n, cplx, "the shifted operator");
        copy_dmat(ctx, sh[k], *as[k]);
        shift_diagonal(ctx, sh[k], -mu_re[k], cplx ? -mu_im[k] : 0.0);
        shp[k] = &sh[k];
    }
    std::vector<double> one_norm = norm1_batch(ctx, shp);

    // The sharp bounds d(p) = normest1(A^p)^(1/p), p = 2..9, for every matrix
    // outside condition 3.13 (:404-410): the search asks for all of them.
    const double scale = std::fabs(t);
    const double ca = 2.0 * kEll * kMaxPower * (kMaxPower + 3);
    const double cb = 9.9 / (ncols * 55.0);
    std::vector<size_t> sharp;
    std::vector<const DMat*> sharp_mats;
    for (size_t k = 0; k < cnt; ++k) {
        const double sn = scale * one_norm[k];
        if (sn != 0.0 && !(sn <= ca * cb)) {
            sharp.push_back(k);
            sharp_mats.push_back(shp[k]);
        }
    }
    std::vector<std::vector<double>> dp(cnt, std::vector<double>(kMaxPower + 2, std::numeric_limits<double>::quiet_NaN()));
    if (!sharp.empty()) {
        // Every (matrix, power) estimator of the batch advances together.
        std::vector<const DMat*> items;
        std::vector<int> powers;
        for (int p = 2; p <= kMaxPower + 1; ++p)
            for (const DMat* m : sharp_mats) {
                items.push_back(m);
                powers.push_back(p);
            }
        std::vector<double> v = power_norm_estimates(ctx, items, powers);
        size_t q = 0;
        for (int p = 2; p <= kMaxPower + 1; ++p)
            for (size_t k = 0; k < sharp.size(); ++k) dp[sharp[k]][p] = std::pow(v[q++], 1.0 / p);
    }

    // (m, s), eta and the coefficients, per matrix (Run, :258-283).
    std::vector<int> ms(cnt), ss(cnt);
    std::vector<double> eta_re(cnt), eta_im(cnt, 0.0);
    std::vector<double> coeffs;
    std::vector<size_t> coeff_off(cnt);
    for (size_t k = 0; k < cnt; ++k) {
        const double sn = scale * one_norm[k];
        int m = 0, s = 1;
        if (sn != 0.0) {
            const std::function<double(int)> alpha = [&](int p) { return net::max(dp[k][p], dp[k][p + 1]); };
            expmv_select_parameters(sn, &alpha, scale, ncols, m, s);
        }
        ms[k] = m;
        ss[k] = s;
        infos[k].degree = m;
        infos[k].scaling = s;
        if (!cplx) {
            eta_re[k] = std::exp((mu_re[k] * t) / (double)s);
        } else {
            net::Cx e = net::exp(net::div(net::Cx{mu_re[k] * t, mu_im[k] * t}, net::Cx{(double)s, 0.0}));
            eta_re[k] = e.re;
            eta_im[k] = e.im;
        }
        coeff_off[k] = coeffs.size();
        for (int j = 0; j < m; ++j) coeffs.push_back(t / (s * (double)(j + 1)));
    }

    if (select_only) return;
    if (ncols > 32) {
        // Wider panels than the fused kernel holds: the host-driven loop.
        for (size_t k = 0; k < cnt; ++k)
            expmv_taylor_host(ctx, sh[k], *bs[k], t, ms[k], ss[k], eta_re[k], eta_im[k], results[k], &infos[k]);
        return;
    }
    // Layout: 8 slots x 64 rows for up to 8 columns, 16 x 32 for up to 16,
    // 16 x 32 with two columns per slot for up to 32.
    const int layout = ncols <= 8 ? 0 : ncols <= 16 ? 1 : 2;
    // The explicit zero skip only when some operator has a non-finite entry
    // (its parameters can still be finite: a nilpotent shifted operator has
    // d(p) = 0 for p >= 2).
    bool skip = false;
    for (size_t k = 0; k < cnt; ++k)
        if (!std::isfinite(one_norm[k])) skip = true;
    const int lanes = taylor(ctx, cplx, skip, layout, nullptr, 0);

    std::vector<int> orders(cnt);
    std::vector<double> apps(cnt);
    for (size_t k = 0; k < cnt; ++k) {
        orders[k] = as[k]->rows;
        apps[k] = std::max(1.0, (double)ms[k] * ss[k]);
    }
    Sched sc = schedule(orders, apps, ncols, lanes, layout == 0 ? 64 : 32);

    std::vector<DMat> w0(cnt), w1(cnt);
    size_t partial_doubles = 0;
    for (size_t k = 0; k < cnt; ++k) {
        results[k] = DMat(ctx, orders[k], ncols, cplx, "the exponential action");
        w0[k] = DMat(ctx, orders[k], ncols, cplx, "a Taylor work panel");
        w1[k] = DMat(ctx, orders[k], ncols, cplx, "a Taylor work panel");
        partial_doubles += 4 * (size_t)sc.width[k];
    }
    const size_t state_bytes = sizeof(unsigned long long) * (cnt + 1) + sizeof(int) * 2 * cnt;
    DBuf state(ctx, state_bytes);
    TNS_CUDA(cudaMemsetAsync(state.p, 0, state_bytes, ctx.stream));
    unsigned long long* bars = state.as<unsigned long long>();
    int* outs = reinterpret_cast<int*>(bars + cnt + 1);
    DBuf partials(ctx, sizeof(double) * std::max<size_t>(partial_doubles, 1));
    DBuf dcoeff(ctx, sizeof(double) * std::max<size_t>(coeffs.size(), 1));
    if (!coeffs.empty())
        TNS_CUDA(cudaMemcpyAsync(dcoeff.p, coeffs.data(), sizeof(double) * coeffs.size(), cudaMemcpyHostToDevice, ctx.stream));
    std::vector<TaylorDesc> descs(cnt);
    size_t poff = 0;
    for (size_t k = 0; k < cnt; ++k) {
        TaylorDesc& d = descs[k];
        d.a = sh[k].p;
        d.lda = sh[k].ld();
        d.b = bs[k]->p;
        d.ldb = bs[k]->ld();
        d.f = results[k].p;
        d.w0 = w0[k].p;
        d.w1 = w1[k].p;
        d.ldp = results[k].ld();
        d.coeff = dcoeff.as<double>() + coeff_off[k];
        d.partials = partials.as<double>() + poff;
        poff += 4 * (size_t)sc.width[k];
        d.bar = bars + k;
        d.out = outs + 2 * k;
        d.n = orders[k];
        d.m = ms[k];
        d.s = ss[k];
        d.width = sc.width[k];
        d.rows_per = sc.rows_per[k];
        d.eta_re = eta_re[k];
        d.eta_im = eta_im[k];
        d.eta_one = (eta_re[k] == 1.0 && eta_im[k] == 0.0) ? 1 : 0;
    }
    TaylorLaunch L{};
    L.descs = static_cast<const TaylorDesc*>(ctx.upload(descs.data(), sizeof(TaylorDesc) * cnt));
    L.plan = static_cast<const TaylorPlan*>(ctx.upload(sc.plan.data(), sizeof(TaylorPlan) * std::max<size_t>(sc.plan.size(), 1)));
    L.plan_off = static_cast<const int*>(ctx.upload(sc.offsets.data(), sizeof(int) * sc.offsets.size()));
    L.ncols = ncols;
    L.err = ctx.d_err;
    L.progress = bars + cnt;
    taylor(ctx, cplx, skip, layout, &L, lanes);
    std::vector<int> h(2 * cnt);
    TNS_CUDA(cudaMemcpyAsync(h.data(), outs, sizeof(int) * 2 * cnt, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    for (size_t k = 0; k < cnt; ++k) {
        infos[k].applications = h[2 * k];
        infos[k].early_exits = h[2 * k + 1];
    }
}

void expmv(Context& ctx, const DMat& a, const DMat& b, double t, DMat& result, ExpmvInfo* info) {
    std::vector<const DMat*> as{&a}, bs{&b};
    std::vector<DMat> res;
    std::vector<ExpmvInfo> infs;
    expmv_batch(ctx, as, bs, t, res, infs);
    result = std::move(res[0]);
    if (info) *info = infs[0];
}

}  // namespace tns
