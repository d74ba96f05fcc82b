// The extern "C" boundary (include/tensile_b200.h). Validates arguments the way
// the reference's KernelEntry / Workspace do, moves operands between the
// caller's buffers and padded device matrices, runs the algorithm, and maps
// internal errors to status codes. Nothing here computes.

#include "tns_internal.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <sstream>
#include <thread>
#include <vector>

struct tns_context {
    tns::Context* impl;
};

namespace {

using tns::Context;
using tns::DMat;
using tns::Error;
using tns::fail;

thread_local std::string g_error_no_ctx;

void check_device_flag(Context& ctx) {
    int h = 0;
    TNS_CUDA(cudaMemcpyAsync(&h, ctx.d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    TNS_CUDA(cudaStreamSynchronize(ctx.stream));
    if (h != 0) {
        TNS_CUDA(cudaMemsetAsync(ctx.d_err, 0, sizeof(int), ctx.stream));
        TNS_CUDA(cudaStreamSynchronize(ctx.stream));
        fail(TNS_E_TIMEOUT, "a device-side wait gave up (code " + std::to_string(h) + ")");
    }
}

template <class F>
int guarded(tns_context* c, F&& body) {
    if (!c || !c->impl) {
        g_error_no_ctx = "The context is null or has been destroyed.";
        return TNS_E_DISPOSED;
    }
    Context& ctx = *c->impl;
    try {
        TNS_CUDA(cudaSetDevice(ctx.device));
        body(ctx);
        check_device_flag(ctx);
        ctx.last_error.clear();
        return TNS_OK;
    } catch (const Error& e) {
        ctx.last_error = e.what();
        // Leave the stream idle so that the caller's buffers may be released.
        cudaStreamSynchronize(ctx.stream);
        return e.code;
    } catch (const std::bad_alloc&) {
        ctx.last_error = "host allocation failed";
        cudaStreamSynchronize(ctx.stream);
        return TNS_E_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        ctx.last_error = e.what();
        cudaStreamSynchronize(ctx.stream);
        return TNS_E_DEVICE;
    }
}

void require(bool cond, int code, const std::string& msg) {
    if (!cond) fail(code, msg);
}

void check_operand(const void* p, int rows, int cols, int ld, const char* name) {
    require(rows >= 0 && cols >= 0, TNS_E_ARGUMENT, std::string(name) + " has a negative dimension");
    require(ld >= std::max(1, rows), TNS_E_ARGUMENT,
            std::string(name) + ": leading dimension " + std::to_string(ld) + " is smaller than its " +
                std::to_string(rows) + " rows");
    require(p != nullptr || (long long)rows * cols == 0, TNS_E_NULL, std::string(name) + " is null");
}

DMat upload(Context& ctx, const double* src, int rows, int cols, int ld, bool cplx, bool on_device, const char* purpose) {
    DMat m(ctx, rows, cols, cplx, purpose);
    tns::copy_in(ctx, m, src, ld, on_device);
    return m;
}

int gemm_entry(tns_context* c, bool cplx, bool dev, int m, int n, int k, const double* alpha, const double* a, int lda,
               const double* b, int ldb, const double* beta, double* cm, int ldc) {
    return guarded(c, [&](Context& ctx) {
        require(alpha != nullptr && beta != nullptr, TNS_E_NULL, "alpha or beta is null");
        check_operand(a, m, k, lda, "A");
        check_operand(b, k, n, ldb, "B");
        check_operand(cm, m, n, ldc, "C");
        if (m == 0 || n == 0) return;
        DMat A = upload(ctx, a, m, k, lda, cplx, dev, "the A operand");
        DMat B = upload(ctx, b, k, n, ldb, cplx, dev, "the B operand");
        bool need_c = !(beta[0] == 0.0 && beta[1] == 0.0);
        DMat C = need_c ? upload(ctx, cm, m, n, ldc, cplx, dev, "the C operand") : DMat(ctx, m, n, cplx, "the C operand");
        if (!cplx && alpha[0] == 0.0) {
            // alpha == 0: C := beta*C only (Gemm.cs:125-127).
            tns::scale_inplace(ctx, C.p, C.rows_p, C.cols_p, C.ld(), false, beta[0], 0.0);
        } else {
            tns::GemmProblem p = tns::make_gemm(A, B, C, alpha[0], alpha[1], beta[0], beta[1]);
            tns::gemm(ctx, p, cplx);
        }
        tns::copy_out(ctx, C, cm, ldc, dev);
        ctx.sync();
    });
}

int gemm_split_entry(tns_context* c, bool cplx, int m, int n, int k, const double* a, int lda, const double* b,
                     int ldb, double* cm, int ldc, int moduli) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, m, k, lda, "A");
        check_operand(b, k, n, ldb, "B");
        check_operand(cm, m, n, ldc, "C");
        require(moduli >= 8 && moduli <= 22, TNS_E_ARGUMENT, "split-precision products take 8 to 22 moduli");
        if (m == 0 || n == 0) return;
        DMat A = upload(ctx, a, m, k, lda, cplx, false, "the A operand");
        DMat B = upload(ctx, b, k, n, ldb, cplx, false, "the B operand");
        DMat C(ctx, m, n, cplx, "the C operand");
        std::vector<tns::SplitProduct> v{tns::SplitProduct{&A, &B, &C, 0.0}};
        tns::gemm_split_batch(ctx, v, moduli);
        tns::copy_out(ctx, C, cm, ldc, false);
        ctx.sync();
    });
}

int norm_entry(tns_context* c, bool cplx, char kind, int m, int n, const double* a, int lda, double* out) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, m, n, lda, "A");
        require(out != nullptr, TNS_E_NULL, "out is null");
        require(kind == '1' || kind == 'I' || kind == 'i' || kind == 'F' || kind == 'f', TNS_E_ARGUMENT,
                "norm kind must be '1', 'I' or 'F'");
        if (m == 0 || n == 0) {
            *out = 0.0;
            return;
        }
        DMat A = upload(ctx, a, m, n, lda, cplx, false, "a norm operand");
        if (kind == '1') *out = tns::norm1(ctx, A);
        else if (kind == 'I' || kind == 'i') *out = tns::norminf(ctx, A);
        else *out = tns::normfro(ctx, A);
    });
}

int getrf_entry(tns_context* c, bool cplx, int m, int n, double* a, int lda, int nb, int* pivots, tns_lu_info* info) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, m, n, lda, "A");
        int limit = std::min(m, n);
        require(pivots != nullptr || limit == 0, TNS_E_NULL, "pivots is null");
        tns_lu_info local{};
        tns_lu_info* out = info ? info : &local;
        *out = tns_lu_info{-1, 0.0, 0.0, 0.0};
        if (limit == 0) return;
        DMat A = upload(ctx, a, m, n, lda, cplx, false, "the matrix to factor");
        // ||A||_1 before factoring (Workspace.cs:214).
        double one = tns::norm1(ctx, A);
        tns::DBuf piv(ctx, sizeof(int) * (size_t)limit);
        tns::LuResult r = tns::getrf(ctx, A, m, n, nb, piv.as<int>());
        std::vector<int> hp(limit);
        TNS_CUDA(cudaMemcpyAsync(hp.data(), piv.p, sizeof(int) * limit, cudaMemcpyDeviceToHost, ctx.stream));
        tns::copy_out(ctx, A, a, lda, false);
        ctx.sync();
        std::memcpy(pivots, hp.data(), sizeof(int) * limit);
        out->singular_column = r.singular_column;
        out->smallest_pivot = r.smallest_pivot;
        out->largest_pivot = r.largest_pivot;
        out->one_norm = one;
    });
}

int getrs_entry(tns_context* c, bool cplx, int n, int nrhs, const double* lu, int lda, const int* pivots,
                int singular_column, double* b, int ldb, int adjoint) {
    return guarded(c, [&](Context& ctx) {
        check_operand(lu, n, n, lda, "the factors");
        check_operand(b, n, nrhs, ldb, "B");
        require(pivots != nullptr || n == 0, TNS_E_NULL, "pivots is null");
        if (singular_column >= 0)
            fail(TNS_E_SINGULAR, "Matrix is singular: zero pivot at column " + std::to_string(singular_column) + ".");
        if (n == 0 || nrhs == 0) return;
        for (int k = 0; k < n; ++k)
            require(pivots[k] >= k && pivots[k] < n, TNS_E_ARGUMENT, "pivot entry out of range");
        DMat F = upload(ctx, lu, n, n, lda, cplx, false, "the factors");
        DMat B = upload(ctx, b, n, nrhs, ldb, cplx, false, "the right-hand sides");
        tns::DBuf piv(ctx, sizeof(int) * (size_t)n);
        TNS_CUDA(cudaMemcpyAsync(piv.p, pivots, sizeof(int) * n, cudaMemcpyHostToDevice, ctx.stream));
        tns::getrs(ctx, F, piv.as<int>(), B, nrhs, adjoint != 0);
        tns::copy_out(ctx, B, b, ldb, false);
        ctx.sync();
    });
}

int gecon_entry(tns_context* c, bool cplx, int n, const double* lu, int lda, const int* pivots, int singular_column,
                double anorm, double* rcond) {
    return guarded(c, [&](Context& ctx) {
        check_operand(lu, n, n, lda, "the factors");
        require(rcond != nullptr, TNS_E_NULL, "rcond is null");
        if (singular_column >= 0 || anorm == 0.0 || n == 0) {
            *rcond = 0.0;
            return;
        }
        require(pivots != nullptr, TNS_E_NULL, "pivots is null");
        for (int k = 0; k < n; ++k)
            require(pivots[k] >= k && pivots[k] < n, TNS_E_ARGUMENT, "pivot entry out of range");
        DMat F = upload(ctx, lu, n, n, lda, cplx, false, "the factors");
        tns::DBuf piv(ctx, sizeof(int) * (size_t)n);
        TNS_CUDA(cudaMemcpyAsync(piv.p, pivots, sizeof(int) * n, cudaMemcpyHostToDevice, ctx.stream));
        tns::NormestResult r = tns::normest_lu_inverse(ctx, F, piv.as<int>(), 2, 5, 20260915);
        *rcond = r.value == 0.0 ? 0.0 : 1.0 / (anorm * r.value);
    });
}

int normest_entry(tns_context* c, bool cplx, int n, const double* a, int lda, int power, int t, int itmax, int seed,
                  tns_normest_result* out) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, n, n, lda, "A");
        require(out != nullptr, TNS_E_NULL, "out is null");
        require(power >= 1, TNS_E_OUT_OF_RANGE, "power must be at least 1");
        *out = tns_normest_result{0.0, 0, 0};
        if (n == 0) return;
        require((long long)n * std::clamp(t, 1, n) <= 2147483647LL, TNS_E_OUT_OF_RANGE, "probe panel too large");
        ctx.check_limit((long long)n * std::clamp(t, 1, n), "an estimator probe panel");
        DMat A = upload(ctx, a, n, n, lda, cplx, false, "the operator");
        tns::NormestResult r = tns::normest_power(ctx, A, power, t, itmax, seed);
        out->value = r.value;
        out->iterations = r.iterations;
        out->products = r.products;
    });
}

// exp of a 1 x 1 matrix: the scalar exponential (MatrixExponential.cs:158-175).
void scalar_exp(const double* a, double* out, bool cplx) {
    if (!cplx) {
        out[0] = std::exp(a[0]);
    } else {
        double e = std::exp(a[0]);
        out[0] = e * std::cos(a[1]);
        out[1] = e * std::sin(a[1]);
    }
}

int expm_entry(tns_context* c, bool cplx, int n, const double* a, int lda, double* out, int ldo, tns_expm_info* info) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, n, n, lda, "A");
        check_operand(out, n, n, ldo, "the result");
        tns_expm_info local{};
        tns_expm_info* inf = info ? info : &local;
        *inf = tns_expm_info{0, 0};
        if (n == 0) return;
        if (n == 1) {
            scalar_exp(a, out, cplx);
            return;
        }
        DMat A = upload(ctx, a, n, n, lda, cplx, false, "the matrix to exponentiate");
        DMat R;
        tns::ExpmInfo ei;
        tns::expm(ctx, A, R, &ei);
        tns::copy_out(ctx, R, out, ldo, false);
        ctx.sync();
        inf->degree = ei.degree;
        inf->squarings = ei.squarings;
    });
}

int expmv_entry(tns_context* c, bool cplx, int n, const double* a, int lda, int ncols, const double* b, int ldb, double t,
                double* out, int ldo, tns_expmv_info* info) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, n, n, lda, "A");
        check_operand(b, n, ncols, ldb, "B");
        check_operand(out, n, ncols, ldo, "the result");
        tns_expmv_info local{};
        tns_expmv_info* inf = info ? info : &local;
        *inf = tns_expmv_info{0, 0, 0, 0};
        if (n == 0 || ncols == 0) return;
        require(std::isfinite(t), TNS_E_OUT_OF_RANGE, "t must be finite");
        DMat A = upload(ctx, a, n, n, lda, cplx, false, "the operator");
        DMat B = upload(ctx, b, n, ncols, ldb, cplx, false, "the panel");
        DMat R;
        tns::ExpmvInfo ei;
        tns::expmv(ctx, A, B, t, R, &ei);
        tns::copy_out(ctx, R, out, ldo, false);
        ctx.sync();
        inf->degree = ei.degree;
        inf->scaling = ei.scaling;
        inf->applications = ei.applications;
        inf->early_exits = ei.early_exits;
    });
}

int expmv_batched_entry(tns_context* c, bool cplx, bool dev, int count, const int* orders, const double* const* a,
                        const int* lda, int ncols, const double* const* b, const int* ldb, double t,
                        double* const* out, const int* ldo, tns_expmv_info* infos) {
    return guarded(c, [&](Context& ctx) {
        require(count >= 0, TNS_E_ARGUMENT, "negative batch size");
        require(ncols >= 0, TNS_E_ARGUMENT, "negative column count");
        if (count == 0) return;
        require(orders && a && lda && b && ldb && out && ldo, TNS_E_NULL, "a batch array is null");
        for (int i = 0; i < count; ++i) {
            check_operand(a[i], orders[i], orders[i], lda[i], "A[i]");
            check_operand(b[i], orders[i], ncols, ldb[i], "B[i]");
            check_operand(out[i], orders[i], ncols, ldo[i], "out[i]");
        }
        require(std::isfinite(t), TNS_E_OUT_OF_RANGE, "t must be finite");
        if (infos)
            for (int i = 0; i < count; ++i) infos[i] = tns_expmv_info{0, 0, 0, 0};
        if (ncols == 0) return;
        std::vector<int> live;
        for (int i = 0; i < count; ++i)
            if (orders[i] > 0) live.push_back(i);
        if (live.empty()) return;
        std::vector<DMat> A, B;
        A.reserve(live.size());
        B.reserve(live.size());
        for (int i : live) {
            A.push_back(upload(ctx, a[i], orders[i], orders[i], lda[i], cplx, dev, "an operator of the batch"));
            B.push_back(upload(ctx, b[i], orders[i], ncols, ldb[i], cplx, dev, "a panel of the batch"));
        }
        std::vector<const DMat*> ap, bp;
        for (size_t k = 0; k < live.size(); ++k) {
            ap.push_back(&A[k]);
            bp.push_back(&B[k]);
        }
        std::vector<DMat> R;
        std::vector<tns::ExpmvInfo> ei;
        tns::expmv_batch(ctx, ap, bp, t, R, ei);
        check_device_flag(ctx);  // a wait that gave up leaves every destination untouched
        for (size_t k = 0; k < live.size(); ++k) tns::copy_out(ctx, R[k], out[live[k]], ldo[live[k]], dev);
        ctx.sync();
        if (infos)
            for (size_t k = 0; k < live.size(); ++k)
                infos[live[k]] = tns_expmv_info{ei[k].degree, ei[k].scaling, ei[k].applications, ei[k].early_exits};
    });
}

// KernelEntry.SolveUpper .. SolveLowerUnitTransposed (KernelEntry.cs:98-173):
// RequireTriangular -- A square, B with A's rows -- then the solve in place.
int trsolve_entry(tns_context* c, bool cplx, tns::TriangularKind kind, int m, int n, const double* a, int lda, double* b,
                  int ldb) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, m, m, lda, "A");
        check_operand(b, m, n, ldb, "B");
        if (m == 0 || n == 0) return;
        DMat A = upload(ctx, a, m, m, lda, cplx, false, "the triangle");
        DMat B = upload(ctx, b, m, n, ldb, cplx, false, "the right-hand sides");
        tns::solve_triangular(ctx, kind, A, B, n);
        check_device_flag(ctx);
        tns::copy_out(ctx, B, b, ldb, false);
        ctx.sync();
    });
}

// KernelEntry.MultiplyPanel / MultiplyPanelTransposed (KernelEntry.cs:176-201):
// RequirePanel -- A square, X and Y n x t -- then Y := A X or A^T X (complex:
// the dense operator's A X or A^H X, LinearOperators.cs:194-293).
int panel_entry(tns_context* c, bool cplx, bool adjoint, int n, int t, const double* a, int lda, const double* x,
                int ldx, double* y, int ldy) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, n, n, lda, "A");
        check_operand(x, n, t, ldx, "X");
        check_operand(y, n, t, ldy, "Y");
        if (n == 0 || t == 0) return;
        DMat A = upload(ctx, a, n, n, lda, cplx, false, "the operator");
        DMat X = upload(ctx, x, n, t, ldx, cplx, false, "the panel");
        DMat Y(ctx, n, t, cplx, "the product panel");
        tns::panel_product(ctx, A, X.p, X.ld(), Y.p, Y.ld(), t, adjoint);
        tns::copy_out(ctx, Y, y, ldy, false);
        ctx.sync();
    });
}

int expmv_select_entry(tns_context* c, bool dev, int count, const int* orders, const double* const* a, const int* lda,
                       int ncols, double t, tns_expmv_info* infos) {
    return guarded(c, [&](Context& ctx) {
        require(count >= 0, TNS_E_ARGUMENT, "negative batch size");
        require(ncols >= 1, TNS_E_ARGUMENT, "the panel needs at least one column");
        if (count == 0) return;
        require(orders && a && lda && infos, TNS_E_NULL, "a batch array is null");
        for (int i = 0; i < count; ++i) check_operand(a[i], orders[i], orders[i], lda[i], "A[i]");
        require(std::isfinite(t), TNS_E_OUT_OF_RANGE, "t must be finite");
        for (int i = 0; i < count; ++i) infos[i] = tns_expmv_info{0, 1, 0, 0};
        std::vector<int> live;
        for (int i = 0; i < count; ++i)
            if (orders[i] > 0) live.push_back(i);
        if (live.empty()) return;
        std::vector<DMat> A;
        A.reserve(live.size());
        for (int i : live) A.push_back(upload(ctx, a[i], orders[i], orders[i], lda[i], true, dev, "an operator of the batch"));
        std::vector<const DMat*> ap;
        for (auto& m : A) ap.push_back(&m);
        std::vector<DMat> R;
        std::vector<tns::ExpmvInfo> ei;
        tns::expmv_batch(ctx, ap, {}, t, R, ei, ncols);
        for (size_t k = 0; k < live.size(); ++k) infos[live[k]] = tns_expmv_info{ei[k].degree, ei[k].scaling, 0, 0};
    });
}

int frechet_entry(tns_context* c, bool cplx, int n, const double* a, int lda, const double* e, int lde, double* expa,
                  int ldx, double* l, int ldl, tns_expm_info* info) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, n, n, lda, "A");
        check_operand(e, n, n, lde, "E");
        check_operand(l, n, n, ldl, "L");
        if (expa) check_operand(expa, n, n, ldx, "exp(A)");
        tns_expm_info local{};
        tns_expm_info* inf = info ? info : &local;
        *inf = tns_expm_info{0, 0};
        if (n == 0) return;
        DMat A = upload(ctx, a, n, n, lda, cplx, false, "the matrix to exponentiate");
        DMat E = upload(ctx, e, n, n, lde, cplx, false, "the direction");
        DMat X, L;
        tns::ExpmInfo ei;
        tns::expm_frechet(ctx, A, E, expa ? &X : nullptr, L, &ei);
        tns::copy_out(ctx, L, l, ldl, false);
        if (expa) tns::copy_out(ctx, X, expa, ldx, false);
        ctx.sync();
        inf->degree = ei.degree;
        inf->squarings = ei.squarings;
    });
}

int gradient_entry(tns_context* c, bool cplx, int n, int nc, double t, const double* a, int lda, const double* b,
                   int ldb, const double* y, int ldy, double* loss, double* ga, int ldga, double* gb, int ldgb,
                   double* gt, double* f, int ldf, tns_expm_info* info) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, n, n, lda, "A");
        check_operand(b, n, nc, ldb, "B");
        check_operand(y, n, nc, ldy, "Y");
        check_operand(ga, n, n, ldga, "dloss/dA");
        check_operand(gb, n, nc, ldgb, "dloss/dB");
        if (f) check_operand(f, n, nc, ldf, "exp(tA) B");
        require(loss != nullptr && gt != nullptr, TNS_E_NULL, "loss or grad_t is null");
        require(std::isfinite(t), TNS_E_OUT_OF_RANGE, "t must be finite");
        tns_expm_info local{};
        tns_expm_info* inf = info ? info : &local;
        *inf = tns_expm_info{0, 0};
        *loss = 0.0;
        *gt = 0.0;
        if (n == 0 || nc == 0) {
            // No entries: zero gradients (an empty B contributes nothing).
            for (int j = 0; j < (nc == 0 ? n : 0); ++j)
                for (int i = 0; i < n; ++i)
                    for (int q = 0; q < (cplx ? 2 : 1); ++q) ga[((size_t)j * ldga + i) * (cplx ? 2 : 1) + q] = 0.0;
            return;
        }
        DMat A = upload(ctx, a, n, n, lda, cplx, false, "the operator");
        DMat B = upload(ctx, b, n, nc, ldb, cplx, false, "the panel");
        DMat Y = upload(ctx, y, n, nc, ldy, cplx, false, "the target");
        DMat F, GA, GB;
        tns::GradientResult r = tns::expmv_gradient(ctx, A, B, Y, t, f ? &F : nullptr, GA, GB);
        tns::copy_out(ctx, GA, ga, ldga, false);
        tns::copy_out(ctx, GB, gb, ldgb, false);
        if (f) tns::copy_out(ctx, F, f, ldf, false);
        ctx.sync();
        *loss = r.loss;
        *gt = r.grad_t;
        inf->degree = r.info.degree;
        inf->squarings = r.info.squarings;
    });
}

int gesv_mixed_entry(tns_context* c, bool cplx, int n, int nrhs, const double* a, int lda, const double* b, int ldb,
                     double* x, int ldx, int moduli, int max_iter, tns_mixed_info* info) {
    return guarded(c, [&](Context& ctx) {
        check_operand(a, n, n, lda, "A");
        check_operand(b, n, nrhs, ldb, "B");
        check_operand(x, n, nrhs, ldx, "X");
        require(moduli == 0 || (moduli >= 8 && moduli <= 22), TNS_E_OUT_OF_RANGE, "moduli must be 0 or 8..22");
        require(max_iter >= 0, TNS_E_OUT_OF_RANGE, "max_iter must not be negative");
        tns_mixed_info local{};
        tns_mixed_info* inf = info ? info : &local;
        *inf = tns_mixed_info{0, 0, 0, 0.0, 0.0, 0};
        if (n == 0 || nrhs == 0) return;
        DMat A = upload(ctx, a, n, n, lda, cplx, false, "the matrix");
        DMat B = upload(ctx, b, n, nrhs, ldb, cplx, false, "the right-hand sides");
        DMat X;
        tns::MixedInfo mi;
        tns::gesv_mixed(ctx, A, B, X, moduli, max_iter, mi);
        tns::copy_out(ctx, X, x, ldx, false);
        ctx.sync();
        *inf = tns_mixed_info{mi.moduli, mi.factorizations, mi.iterations, mi.backward_error, mi.rcond, mi.pivoting};
    });
}

int normest_operator_entry(tns_context* c, bool cplx, int n, tns_apply_fn apply, tns_apply_fn adjoint, void* user,
                           int t, int itmax, int seed, tns_normest_result* out) {
    return guarded(c, [&](Context& ctx) {
        require(apply != nullptr && adjoint != nullptr, TNS_E_NULL, "The operator is null.");
        require(out != nullptr, TNS_E_NULL, "out is null");
        require(n >= 0, TNS_E_ARGUMENT, "negative order");
        *out = tns_normest_result{0.0, 0, 0};
        if (n == 0) return;
        require((long long)n * std::clamp(t, 1, n) <= 2147483647LL, TNS_E_OUT_OF_RANGE, "probe panel too large");
        ctx.check_limit((long long)n * std::clamp(t, 1, n), "an estimator probe panel");
        tns::NormestResult r = tns::normest_operator(ctx, n, cplx, apply, adjoint, user, t, itmax, seed);
        out->value = r.value;
        out->iterations = r.iterations;
        out->products = r.products;
    });
}

int expmv_operator_entry(tns_context* c, bool cplx, int n, tns_apply_fn apply, void* user, int ncols,
                         const double* b, int ldb, double t, double bound, double* out, int ldo, tns_expmv_info* info) {
    return guarded(c, [&](Context& ctx) {
        require(apply != nullptr, TNS_E_NULL, "The operator is null.");
        check_operand(b, n, ncols, ldb, "B");
        check_operand(out, n, ncols, ldo, "the result");
        require(std::isfinite(bound) && bound >= 0.0, TNS_E_OUT_OF_RANGE,
                "The norm bound must be finite and not negative.");
        require(std::isfinite(t), TNS_E_OUT_OF_RANGE, "t must be finite");
        tns_expmv_info local{};
        tns_expmv_info* inf = info ? info : &local;
        *inf = tns_expmv_info{0, 0, 0, 0};
        if (n == 0 || ncols == 0) return;
        DMat B = upload(ctx, b, n, ncols, ldb, cplx, false, "the panel");
        DMat R;
        tns::ExpmvInfo ei;
        tns::expmv_operator(ctx, n, apply, user, B, t, bound, R, &ei);
        tns::copy_out(ctx, R, out, ldo, false);
        ctx.sync();
        inf->degree = ei.degree;
        inf->scaling = ei.scaling;
        inf->applications = ei.applications;
        inf->early_exits = ei.early_exits;
    });
}

// True for page-locked host memory (cudaHostAlloc / cudaHostRegister).
bool host_pinned(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

int zexpm_batched_entry(tns_context* c, bool dev, int count, const int* orders, const double* const* a, const int* lda,
                        double* const* out, const int* ldo, tns_expm_info* infos) {
    return guarded(c, [&](Context& ctx) {
        require(count >= 0, TNS_E_ARGUMENT, "negative batch size");
        if (count == 0) return;
        require(orders && a && lda && out && ldo, TNS_E_NULL, "a batch array is null");
        for (int i = 0; i < count; ++i) {
            check_operand(a[i], orders[i], orders[i], lda[i], "A[i]");
            check_operand(out[i], orders[i], orders[i], ldo[i], "out[i]");
        }
        std::vector<tns_expm_info> results(count, tns_expm_info{0, 0});
        // Orders 0 and 1 need no device work (MatrixExponential.cs:158-175).
        std::vector<int> big;
        for (int i = 0; i < count; ++i) {
            int n = orders[i];
            if (n >= 2) {
                big.push_back(i);
            } else if (n == 1) {
                double h[2], r[2];
                if (dev) {
                    TNS_CUDA(cudaMemcpyAsync(h, a[i], 16, cudaMemcpyDeviceToHost, ctx.stream));
                    ctx.sync();
                    scalar_exp(h, r, true);
                    TNS_CUDA(cudaMemcpyAsync(out[i], r, 16, cudaMemcpyHostToDevice, ctx.stream));
                    ctx.sync();
                } else {
                    scalar_exp(a[i], out[i], true);
                }
            }
        }
        // Split the rest into cost-balanced groups (largest first onto the
        // lightest group, n^3 as the cost); each group runs the batched
        // algorithm on its own worker stream, so one group's host-side
        // decisions and copies overlap another group's kernels.
        int ngroups = std::max(1, std::min((int)big.size(), ctx.max_workers));
        std::stable_sort(big.begin(), big.end(), [&](int x, int y) { return orders[x] > orders[y]; });
        std::vector<std::vector<int>> groups(ngroups);
        std::vector<double> load(ngroups, 0.0);
        for (int i : big) {
            int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            groups[g].push_back(i);
            load[g] += std::pow((double)orders[i], 3.0);
        }
        int nworkers = ngroups;
        // Host inputs: the groups' copies in take turns (group w's after group
        // w - 1's, ordered by an event), so that the first group computes
        // while the others' matrices are still crossing instead of every
        // group waiting for all the copies at once.
        std::vector<cudaEvent_t> uploaded(nworkers, nullptr);
        std::vector<char> recorded(nworkers, 0);
        std::mutex turn_mu;
        std::condition_variable turn_cv;
        if (!dev && nworkers > 1)
            for (auto& e : uploaded) TNS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        auto mark_recorded = [&](int w) {
            std::lock_guard<std::mutex> g(turn_mu);
            recorded[w] = 1;
            turn_cv.notify_all();
        };
        auto run_group = [&](Context& wc, const std::vector<int>& idx, int w) {
            const bool turns = !dev && nworkers > 1;
            if (turns && w > 0) {
                std::unique_lock<std::mutex> g(turn_mu);
                turn_cv.wait(g, [&] { return recorded[w - 1] != 0; });
                g.unlock();
                TNS_CUDA(cudaStreamWaitEvent(wc.stream, uploaded[w - 1], 0));
            }
            std::vector<DMat> in;
            in.reserve(idx.size());
            for (int i : idx) in.push_back(upload(wc, a[i], orders[i], orders[i], lda[i], true, dev, "a matrix to exponentiate"));
            if (turns) {
                TNS_CUDA(cudaEventRecord(uploaded[w], wc.stream));
                mark_recorded(w);
            }
            if (idx.empty()) return;
            std::vector<const DMat*> ptrs;
            for (auto& m : in) ptrs.push_back(&m);
            std::vector<DMat> res;
            std::vector<tns::ExpmInfo> infs;
            const bool early = !dev && std::all_of(idx.begin(), idx.end(), [&](int i) { return host_pinned(out[i]); });
            if (!early) {
                tns::expm_batch(wc, ptrs, res, infs);
                for (size_t k = 0; k < idx.size(); ++k) tns::copy_out(wc, res[k], out[idx[k]], ldo[idx[k]], dev);
            } else {
                // Pinned host outputs: each result crosses to the host on the
                // copy stream as soon as it is final, while the group's other
                // matrices still square. (A copy into pageable memory would
                // hold this thread until the copy ran, so those results go at
                // the end.) The results outlive the fence, whose destructor,
                // on every path, orders their frees on the group's stream
                // after the copies.
                std::vector<DMat> finished(idx.size());
                cudaStream_t cs = wc.copies();
                cudaEvent_t ready = nullptr;
                TNS_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
                struct CopyFence {
                    Context& wc;
                    cudaStream_t cs;
                    cudaEvent_t ev;
                    ~CopyFence() {
                        cudaEventRecord(ev, cs);
                        cudaStreamWaitEvent(wc.stream, ev, 0);
                        cudaStreamSynchronize(wc.stream);
                        cudaEventDestroy(ev);
                    }
                } fence{wc, cs, ready};
                tns::expm_batch(wc, ptrs, res, infs, [&](size_t k, DMat&& r) {
                    finished[k] = std::move(r);
                    TNS_CUDA(cudaEventRecord(ready, wc.stream));
                    TNS_CUDA(cudaStreamWaitEvent(cs, ready, 0));
                    tns::copy_out_on(cs, finished[k], out[idx[k]], ldo[idx[k]], false);
                });
            }
            for (size_t k = 0; k < idx.size(); ++k)
                results[idx[k]] = tns_expm_info{infs[k].degree, infs[k].squarings};
            wc.sync();
        };

        while ((int)ctx.workers.size() < nworkers) ctx.workers.emplace_back(new Context(ctx.device));
        std::atomic<bool> stop{false};
        std::mutex mu;
        int err_code = TNS_OK;
        std::string err_msg;
        auto worker = [&](int w) {
            Context& wc = *ctx.workers[w];
            wc.max_elements = ctx.max_elements;
            wc.timing = ctx.timing;
            wc.split_moduli = ctx.split_moduli;
            wc.autotune = ctx.autotune;
            wc.concurrent = true;
            try {
                TNS_CUDA(cudaSetDevice(ctx.device));
                run_group(wc, groups[w], w);
                check_device_flag(wc);
            } catch (const Error& e) {
                std::lock_guard<std::mutex> g(mu);
                if (err_code == TNS_OK) {
                    err_code = e.code;
                    err_msg = e.what();
                }
                stop = true;
                cudaStreamSynchronize(wc.stream);
            } catch (const std::exception& e) {
                std::lock_guard<std::mutex> g(mu);
                if (err_code == TNS_OK) {
                    err_code = TNS_E_DEVICE;
                    err_msg = e.what();
                }
                stop = true;
                cudaStreamSynchronize(wc.stream);
            }
        };
        // A worker that stops early still lets the next one take its turn.
        auto worker_turn = [&](int w) {
            worker(w);
            mark_recorded(w);
        };
        if (nworkers == 1) {
            worker_turn(0);
        } else {
            std::vector<std::thread> threads;
            threads.reserve(nworkers);
            for (int w = 0; w < nworkers; ++w) threads.emplace_back(worker_turn, w);
            for (auto& th : threads) th.join();
        }
        for (auto& e : uploaded)
            if (e) cudaEventDestroy(e);
        if (err_code != TNS_OK) fail(err_code, err_msg);
        if (infos)
            for (int i = 0; i < count; ++i) infos[i] = results[i];
    });
}

// Sum of a context's counters and those of its batch workers.
void collect_stats(Context& ctx, tns_stats* out) {
    ctx.drain_events();
    out->kernel_launches = ctx.kernel_launches;
    out->gemm_launches = ctx.gemm_launches;
    out->gemm_flops = ctx.gemm_flops;
    out->gemm_ms = ctx.gemm_ms_done;
    out->gemm_bytes = ctx.gemm_bytes;
    out->split_launches = ctx.split_launches;
    out->split_flops = ctx.split_flops;
    out->split_int8_ops = ctx.split_int8_ops;
    out->split_ms = ctx.split_ms_done;
    out->split_bytes = ctx.split_bytes;
    out->autotune_trials = ctx.autotune_trials;
    out->exact_fallbacks = ctx.exact_fallbacks;
    for (auto& w : ctx.workers) {
        w->drain_events();
        out->kernel_launches += w->kernel_launches;
        out->gemm_launches += w->gemm_launches;
        out->gemm_flops += w->gemm_flops;
        out->gemm_ms += w->gemm_ms_done;
        out->gemm_bytes += w->gemm_bytes;
        out->split_launches += w->split_launches;
        out->split_flops += w->split_flops;
        out->split_int8_ops += w->split_int8_ops;
        out->split_ms += w->split_ms_done;
        out->split_bytes += w->split_bytes;
        out->autotune_trials += w->autotune_trials;
        out->exact_fallbacks += w->exact_fallbacks;
    }
}

void reset_stats(Context& ctx) {
    ctx.drain_events();
    ctx.kernel_launches = ctx.gemm_launches = 0;
    ctx.gemm_flops = ctx.gemm_ms_done = ctx.gemm_bytes = 0.0;
    ctx.split_launches = 0;
    ctx.split_flops = ctx.split_int8_ops = ctx.split_ms_done = ctx.split_bytes = 0.0;
    ctx.autotune_trials = 0;
    ctx.exact_fallbacks = 0;
    ctx.lu_panel_ms = ctx.lu_swaps_ms = ctx.lu_triangular_ms = ctx.lu_gemm_ms = ctx.lu_total_ms = 0.0;
    ctx.lu_block_steps = ctx.lu_factorizations = 0;
    for (auto& w : ctx.workers) {
        w->drain_events();
        w->kernel_launches = w->gemm_launches = 0;
        w->gemm_flops = w->gemm_ms_done = w->gemm_bytes = 0.0;
        w->split_launches = 0;
        w->split_flops = w->split_int8_ops = w->split_ms_done = w->split_bytes = 0.0;
        w->autotune_trials = 0;
        w->exact_fallbacks = 0;
    }
}

}  // namespace

void tns::set_detached_error(const std::string& msg) { g_error_no_ctx = msg; }

extern "C" {

int tns_create(int device, long long max_elements, tns_context** out) {
    if (!out) return TNS_E_NULL;
    *out = nullptr;
    try {
        auto* c = new tns_context{new Context(device)};
        if (max_elements > 0) c->impl->max_elements = std::min(max_elements, 2147483591LL);
        *out = c;
        return TNS_OK;
    } catch (const Error& e) {
        g_error_no_ctx = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_error_no_ctx = e.what();
        return TNS_E_DEVICE;
    }
}

int tns_destroy(tns_context* ctx) {
    if (!ctx) return TNS_E_DISPOSED;
    delete ctx->impl;
    ctx->impl = nullptr;
    delete ctx;
    return TNS_OK;
}

const char* tns_last_error(const tns_context* ctx) {
    if (!ctx || !ctx->impl) return g_error_no_ctx.c_str();
    return ctx->impl->last_error.c_str();
}

int tns_set_max_elements(tns_context* ctx, long long max_elements) {
    return guarded(ctx, [&](Context& c) {
        require(max_elements > 0 && max_elements <= 2147483591LL, TNS_E_OUT_OF_RANGE,
                "MaxElements must be positive and at most Array.MaxLength");
        c.max_elements = max_elements;
    });
}

int tns_dgemm(tns_context* c, int m, int n, int k, double alpha, const double* a, int lda, const double* b, int ldb,
              double beta, double* cm, int ldc) {
    double al[2] = {alpha, 0.0}, be[2] = {beta, 0.0};
    return gemm_entry(c, false, false, m, n, k, al, a, lda, b, ldb, be, cm, ldc);
}
int tns_dgemm_device(tns_context* c, int m, int n, int k, double alpha, const double* a, int lda, const double* b,
                     int ldb, double beta, double* cm, int ldc) {
    double al[2] = {alpha, 0.0}, be[2] = {beta, 0.0};
    return gemm_entry(c, false, true, m, n, k, al, a, lda, b, ldb, be, cm, ldc);
}
int tns_zgemm(tns_context* c, int m, int n, int k, const double* alpha, const double* a, int lda, const double* b,
              int ldb, const double* beta, double* cm, int ldc) {
    return gemm_entry(c, true, false, m, n, k, alpha, a, lda, b, ldb, beta, cm, ldc);
}
int tns_zgemm_device(tns_context* c, int m, int n, int k, const double* alpha, const double* a, int lda,
                     const double* b, int ldb, const double* beta, double* cm, int ldc) {
    return gemm_entry(c, true, true, m, n, k, alpha, a, lda, b, ldb, beta, cm, ldc);
}

int tns_dgemm_split(tns_context* c, int m, int n, int k, const double* a, int lda, const double* b, int ldb,
                    double* cm, int ldc, int moduli) {
    return gemm_split_entry(c, false, m, n, k, a, lda, b, ldb, cm, ldc, moduli);
}
int tns_zgemm_split(tns_context* c, int m, int n, int k, const double* a, int lda, const double* b, int ldb,
                    double* cm, int ldc, int moduli) {
    return gemm_split_entry(c, true, m, n, k, a, lda, b, ldb, cm, ldc, moduli);
}
int tns_set_split_moduli(tns_context* c, int moduli) {
    return guarded(c, [&](Context& ctx) {
        require(moduli == 0 || (moduli >= 8 && moduli <= 22), TNS_E_ARGUMENT,
                "split moduli must be 0 (plain FP64) or 8 to 22");
        ctx.split_moduli = moduli;
        for (auto& w : ctx.workers) w->split_moduli = moduli;
    });
}

int tns_dnorm(tns_context* c, char kind, int m, int n, const double* a, int lda, double* out) {
    return norm_entry(c, false, kind, m, n, a, lda, out);
}
int tns_znorm(tns_context* c, char kind, int m, int n, const double* a, int lda, double* out) {
    return norm_entry(c, true, kind, m, n, a, lda, out);
}

int tns_dgetrf(tns_context* c, int m, int n, double* a, int lda, int nb, int* pivots, tns_lu_info* info) {
    return getrf_entry(c, false, m, n, a, lda, nb, pivots, info);
}
int tns_zgetrf(tns_context* c, int m, int n, double* a, int lda, int nb, int* pivots, tns_lu_info* info) {
    return getrf_entry(c, true, m, n, a, lda, nb, pivots, info);
}
int tns_dgetrs(tns_context* c, int n, int nrhs, const double* lu, int lda, const int* pivots, int singular_column,
               double* b, int ldb, int adjoint) {
    return getrs_entry(c, false, n, nrhs, lu, lda, pivots, singular_column, b, ldb, adjoint);
}
int tns_zgetrs(tns_context* c, int n, int nrhs, const double* lu, int lda, const int* pivots, int singular_column,
               double* b, int ldb, int adjoint) {
    return getrs_entry(c, true, n, nrhs, lu, lda, pivots, singular_column, b, ldb, adjoint);
}
int tns_dgecon(tns_context* c, int n, const double* lu, int lda, const int* pivots, int singular_column, double anorm,
               double* rcond) {
    return gecon_entry(c, false, n, lu, lda, pivots, singular_column, anorm, rcond);
}
int tns_zgecon(tns_context* c, int n, const double* lu, int lda, const int* pivots, int singular_column, double anorm,
               double* rcond) {
    return gecon_entry(c, true, n, lu, lda, pivots, singular_column, anorm, rcond);
}
int tns_dnormest1_power(tns_context* c, int n, const double* a, int lda, int power, int t, int itmax, int seed,
                        tns_normest_result* out) {
    return normest_entry(c, false, n, a, lda, power, t, itmax, seed, out);
}
int tns_znormest1_power(tns_context* c, int n, const double* a, int lda, int power, int t, int itmax, int seed,
                        tns_normest_result* out) {
    return normest_entry(c, true, n, a, lda, power, t, itmax, seed, out);
}
int tns_dexpm(tns_context* c, int n, const double* a, int lda, double* out, int ldo, tns_expm_info* info) {
    return expm_entry(c, false, n, a, lda, out, ldo, info);
}
int tns_zexpm(tns_context* c, int n, const double* a, int lda, double* out, int ldo, tns_expm_info* info) {
    return expm_entry(c, true, n, a, lda, out, ldo, info);
}
int tns_zexpm_batched(tns_context* c, int count, const int* orders, const double* const* a, const int* lda,
                      double* const* out, const int* ldo, tns_expm_info* infos) {
    return zexpm_batched_entry(c, false, count, orders, a, lda, out, ldo, infos);
}
int tns_zexpm_batched_device(tns_context* c, int count, const int* orders, const double* const* a, const int* lda,
                             double* const* out, const int* ldo, tns_expm_info* infos) {
    return zexpm_batched_entry(c, true, count, orders, a, lda, out, ldo, infos);
}
#define TNS_TRSOLVE(name, cplx, kind)                                                                  \
    int name(tns_context* c, int m, int n, const double* a, int lda, double* b, int ldb) {                \
        return trsolve_entry(c, cplx, tns::TriangularKind::kind, m, n, a, lda, b, ldb);                   \
    }
TNS_TRSOLVE(tns_dsolve_upper, false, kUpper)
TNS_TRSOLVE(tns_dsolve_upper_transposed, false, kUpperTransposed)
TNS_TRSOLVE(tns_dsolve_lower, false, kLower)
TNS_TRSOLVE(tns_dsolve_lower_transposed, false, kLowerTransposed)
TNS_TRSOLVE(tns_dsolve_lower_unit, false, kLowerUnit)
TNS_TRSOLVE(tns_dsolve_lower_unit_transposed, false, kLowerUnitTransposed)
TNS_TRSOLVE(tns_zsolve_upper, true, kUpper)
TNS_TRSOLVE(tns_zsolve_upper_adjoint, true, kUpperTransposed)
TNS_TRSOLVE(tns_zsolve_lower_unit, true, kLowerUnit)
TNS_TRSOLVE(tns_zsolve_lower_unit_adjoint, true, kLowerUnitTransposed)
#undef TNS_TRSOLVE

int tns_dmultiply_panel(tns_context* c, int n, int t, const double* a, int lda, const double* x, int ldx, double* y,
                        int ldy) {
    return panel_entry(c, false, false, n, t, a, lda, x, ldx, y, ldy);
}
int tns_dmultiply_panel_transposed(tns_context* c, int n, int t, const double* a, int lda, const double* x, int ldx,
                                   double* y, int ldy) {
    return panel_entry(c, false, true, n, t, a, lda, x, ldx, y, ldy);
}
int tns_zmultiply_panel(tns_context* c, int n, int t, const double* a, int lda, const double* x, int ldx, double* y,
                        int ldy) {
    return panel_entry(c, true, false, n, t, a, lda, x, ldx, y, ldy);
}
int tns_zmultiply_panel_adjoint(tns_context* c, int n, int t, const double* a, int lda, const double* x, int ldx,
                                double* y, int ldy) {
    return panel_entry(c, true, true, n, t, a, lda, x, ldx, y, ldy);
}

int tns_dexpmv_batched(tns_context* c, int count, const int* orders, const double* const* a, const int* lda, int ncols,
                       const double* const* b, const int* ldb, double t, double* const* out, const int* ldo,
                       tns_expmv_info* infos) {
    return expmv_batched_entry(c, false, false, count, orders, a, lda, ncols, b, ldb, t, out, ldo, infos);
}
int tns_zexpmv_batched(tns_context* c, int count, const int* orders, const double* const* a, const int* lda, int ncols,
                       const double* const* b, const int* ldb, double t, double* const* out, const int* ldo,
                       tns_expmv_info* infos) {
    return expmv_batched_entry(c, true, false, count, orders, a, lda, ncols, b, ldb, t, out, ldo, infos);
}
int tns_zexpmv_batched_device(tns_context* c, int count, const int* orders, const double* const* a, const int* lda,
                              int ncols, const double* const* b, const int* ldb, double t, double* const* out,
                              const int* ldo, tns_expmv_info* infos) {
    return expmv_batched_entry(c, true, true, count, orders, a, lda, ncols, b, ldb, t, out, ldo, infos);
}
int tns_zexpmv_select_batched(tns_context* c, int count, const int* orders, const double* const* a, const int* lda,
                              int ncols, double t, tns_expmv_info* infos) {
    return expmv_select_entry(c, false, count, orders, a, lda, ncols, t, infos);
}
int tns_zexpmv_select_batched_device(tns_context* c, int count, const int* orders, const double* const* a,
                                     const int* lda, int ncols, double t, tns_expmv_info* infos) {
    return expmv_select_entry(c, true, count, orders, a, lda, ncols, t, infos);
}
int tns_dexpm_frechet(tns_context* c, int n, const double* a, int lda, const double* e, int lde, double* expa,
                      int ldx, double* l, int ldl, tns_expm_info* info) {
    return frechet_entry(c, false, n, a, lda, e, lde, expa, ldx, l, ldl, info);
}
int tns_zexpm_frechet(tns_context* c, int n, const double* a, int lda, const double* e, int lde, double* expa,
                      int ldx, double* l, int ldl, tns_expm_info* info) {
    return frechet_entry(c, true, n, a, lda, e, lde, expa, ldx, l, ldl, info);
}
int tns_dexpmv_gradient(tns_context* c, int n, int ncols, double t, const double* a, int lda, const double* b,
                        int ldb, const double* y, int ldy, double* loss, double* grad_a, int ldga, double* grad_b,
                        int ldgb, double* grad_t, double* f, int ldf, tns_expm_info* info) {
    return gradient_entry(c, false, n, ncols, t, a, lda, b, ldb, y, ldy, loss, grad_a, ldga, grad_b, ldgb, grad_t, f,
                          ldf, info);
}
int tns_zexpmv_gradient(tns_context* c, int n, int ncols, double t, const double* a, int lda, const double* b,
                        int ldb, const double* y, int ldy, double* loss, double* grad_a, int ldga, double* grad_b,
                        int ldgb, double* grad_t, double* f, int ldf, tns_expm_info* info) {
    return gradient_entry(c, true, n, ncols, t, a, lda, b, ldb, y, ldy, loss, grad_a, ldga, grad_b, ldgb, grad_t, f,
                          ldf, info);
}
int tns_dnormest1_operator(tns_context* c, int n, tns_apply_fn apply, tns_apply_fn adjoint, void* user, int t,
                           int itmax, int seed, tns_normest_result* out) {
    return normest_operator_entry(c, false, n, apply, adjoint, user, t, itmax, seed, out);
}
int tns_znormest1_operator(tns_context* c, int n, tns_apply_fn apply, tns_apply_fn adjoint, void* user, int t,
                           int itmax, int seed, tns_normest_result* out) {
    return normest_operator_entry(c, true, n, apply, adjoint, user, t, itmax, seed, out);
}
int tns_dexpmv_operator(tns_context* c, int n, tns_apply_fn apply, void* user, int ncols, const double* b, int ldb,
                        double t, double one_norm_bound, double* out, int ldo, tns_expmv_info* info) {
    return expmv_operator_entry(c, false, n, apply, user, ncols, b, ldb, t, one_norm_bound, out, ldo, info);
}
int tns_zexpmv_operator(tns_context* c, int n, tns_apply_fn apply, void* user, int ncols, const double* b, int ldb,
                        double t, double one_norm_bound, double* out, int ldo, tns_expmv_info* info) {
    return expmv_operator_entry(c, true, n, apply, user, ncols, b, ldb, t, one_norm_bound, out, ldo, info);
}
int tns_dgesv_mixed(tns_context* c, int n, int nrhs, const double* a, int lda, const double* b, int ldb, double* x,
                    int ldx, int moduli, int max_iter, tns_mixed_info* info) {
    return gesv_mixed_entry(c, false, n, nrhs, a, lda, b, ldb, x, ldx, moduli, max_iter, info);
}
int tns_zgesv_mixed(tns_context* c, int n, int nrhs, const double* a, int lda, const double* b, int ldb, double* x,
                    int ldx, int moduli, int max_iter, tns_mixed_info* info) {
    return gesv_mixed_entry(c, true, n, nrhs, a, lda, b, ldb, x, ldx, moduli, max_iter, info);
}
int tns_set_autotune(tns_context* c, int enabled) {
    return guarded(c, [&](Context& ctx) {
        ctx.autotune = enabled != 0;
        for (auto& w : ctx.workers) w->autotune = ctx.autotune;
    });
}
int tns_set_checkpoint_bytes(tns_context* c, long long bytes) {
    return guarded(c, [&](Context& ctx) {
        require(bytes >= -1, TNS_E_OUT_OF_RANGE, "checkpoint bytes must be -1 (automatic) or a byte count");
        ctx.checkpoint_bytes = bytes;
    });
}
int tns_get_stats(tns_context* c, tns_stats* out) {
    return guarded(c, [&](Context& ctx) {
        require(out != nullptr, TNS_E_NULL, "out is null");
        collect_stats(ctx, out);
    });
}
int tns_reset_stats(tns_context* c) {
    return guarded(c, [&](Context& ctx) { reset_stats(ctx); });
}
int tns_set_workers(tns_context* c, int workers) {
    return guarded(c, [&](Context& ctx) {
        require(workers >= 1 && workers <= 128, TNS_E_OUT_OF_RANGE, "workers must be in [1, 128]");
        ctx.max_workers = workers;
    });
}
int tns_set_timing(tns_context* c, int enabled) {
    return guarded(c, [&](Context& ctx) { ctx.timing = enabled != 0; });
}
int tns_inject_allocation_failure(tns_context* c, long long k) {
    return guarded(c, [&](Context& ctx) {
        require(k >= 0, TNS_E_OUT_OF_RANGE, "k must be >= 0");
        ctx.fail_allocation_at = k > 0 ? ctx.allocations + k : 0;
    });
}
int tns_selftest_wait(tns_context* c, long long limit_ns) {
    return guarded(c, [&](Context& ctx) {
        require(limit_ns > 0 && limit_ns <= 2000000000LL, TNS_E_OUT_OF_RANGE, "limit_ns must be in (0, 2e9]");
        tns::selftest_wait(ctx, limit_ns);
    });
}
int tns_set_lu_timing(tns_context* c, int enabled) {
    return guarded(c, [&](Context& ctx) { ctx.lu_timing = enabled != 0; });
}
int tns_get_lu_timings(tns_context* c, tns_lu_timings* out) {
    return guarded(c, [&](Context& ctx) {
        require(out != nullptr, TNS_E_NULL, "out is null");
        out->panel_ms = ctx.lu_panel_ms;
        out->swaps_ms = ctx.lu_swaps_ms;
        out->triangular_ms = ctx.lu_triangular_ms;
        out->gemm_ms = ctx.lu_gemm_ms;
        out->total_ms = ctx.lu_total_ms;
        // The residue the phases do not account for, never negative
        // (LuPhaseTimings.Unattributed).
        out->unattributed_ms = std::max(0.0, ctx.lu_total_ms - (ctx.lu_panel_ms + ctx.lu_swaps_ms +
                                                                  ctx.lu_triangular_ms + ctx.lu_gemm_ms));
        out->block_steps = ctx.lu_block_steps;
        out->factorizations = ctx.lu_factorizations;
    });
}
int tns_get_stream(tns_context* c, void** stream) {
    return guarded(c, [&](Context& ctx) {
        require(stream != nullptr, TNS_E_NULL, "stream is null");
        *stream = reinterpret_cast<void*>(ctx.stream);
    });
}

int tns_dexpmv(tns_context* c, int n, const double* a, int lda, int ncols, const double* b, int ldb, double t,
               double* out, int ldo, tns_expmv_info* info) {
    return expmv_entry(c, false, n, a, lda, ncols, b, ldb, t, out, ldo, info);
}
int tns_zexpmv(tns_context* c, int n, const double* a, int lda, int ncols, const double* b, int ldb, double t,
               double* out, int ldo, tns_expmv_info* info) {
    return expmv_entry(c, true, n, a, lda, ncols, b, ldb, t, out, ldo, info);
}

}  // extern "C"
