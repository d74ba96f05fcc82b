/*
 * tensile_b200 -- C ABI of the B200-native (sm_100a) dense hot path of the
 * Tensile linear algebra library.
 *
 * Every entry point replaces a computation the reference library performs in
 * managed C# behind its kernel seam (src/Tensile.Kernels/KernelEntry.cs:31-270)
 * or, for whole algorithms, in src/Tensile (complex products, LU of complex
 * matrices, normest1, Expm, Expmv). Each declaration names the reference
 * interface it stands in for (paths relative to the reference project root).
 *
 * Conventions
 *  - Matrices are column-major with a leading dimension (ld >= rows, counted
 *    in elements), as MatrixShape defines them (src/Tensile/MatrixShape.cs:20-152).
 *  - Complex matrices are interleaved (re, im) pairs of doubles: the memory
 *    layout of System.Numerics.Complex, so a pinned Complex[] passes as is.
 *  - Host-pointer entry points are synchronous: they copy the operands to the
 *    GPU, compute, copy the results back and return only when the host buffers
 *    may be unpinned (the reference pins spans for exactly one call,
 *    src/Tensile.Kernels/KernelEntry.cs:3-30). On failure the destination is
 *    left untouched (src/Tensile/ComplexKernels.cs:103-106).
 *  - Entry points ending in _device take device pointers instead and run on the
 *    context's stream; they also return only when the work has finished.
 *  - Calls on one context are serialised (one CUDA stream per context, as one
 *    Workspace serialises its operations on one lock,
 *    src/Tensile/Workspace.cs:42,136-139). Distinct contexts are independent.
 *  - Return value: TNS_OK or one of the TNS_E_* codes below; tns_last_error()
 *    gives the message. The codes map one to one onto the exceptions the
 *    reference throws for the same conditions.
 */
#ifndef TENSILE_B200_H
#define TENSILE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define TNS_OK 0
#define TNS_E_ARGUMENT 1         /* ArgumentException: shapes disagree, bad ld, not square */
#define TNS_E_SINGULAR 2         /* InvalidOperationException: exactly zero pivot */
#define TNS_E_ALLOCATION_LIMIT 3 /* AllocationLimitException (src/Tensile/TensileLimits.cs:59-96) */
#define TNS_E_OUT_OF_MEMORY 4    /* device allocation failed */
#define TNS_E_DEVICE 5           /* CUDA runtime error */
#define TNS_E_TIMEOUT 6          /* a bounded device-side wait gave up */
#define TNS_E_DISPOSED 7         /* ObjectDisposedException: null or destroyed context */
#define TNS_E_OUT_OF_RANGE 8     /* ArgumentOutOfRangeException */
#define TNS_E_NULL 9             /* ArgumentNullException */
#define TNS_E_OPERATOR 10        /* a caller's operator callback reported failure */

typedef struct tns_context tns_context;

/* Workspace(multithreaded) construction and Dispose (src/Tensile/Workspace.cs:52-72, 252-262):
 * one CUDA stream and the device buffers of one workspace. max_elements is
 * TensileLimits.MaxElements (src/Tensile/TensileLimits.cs:27-65); <= 0 means
 * the reference default, Array.MaxLength. */
int tns_create(int device, long long max_elements, tns_context** out);
int tns_destroy(tns_context* ctx);
const char* tns_last_error(const tns_context* ctx);
int tns_set_max_elements(tns_context* ctx, long long max_elements);

/* ---- products ----------------------------------------------------------- */

/* C := beta*C + alpha*A*B, A m x k, B k x n. beta == 0 overwrites C (NaN in C
 * does not survive). KernelEntry.Multiply (src/Tensile.Kernels/KernelEntry.cs:34-56)
 * -> Gemm/ParallelGemm (src/Tensile.Kernels/Gemm.cs:117-203). */
int tns_dgemm(tns_context* ctx, int m, int n, int k, double alpha, const double* a, int lda,
              const double* b, int ldb, double beta, double* c, int ldc);
int tns_dgemm_device(tns_context* ctx, int m, int n, int k, double alpha, const double* a, int lda,
                     const double* b, int ldb, double beta, double* c, int ldc);

/* Complex C := beta*C + alpha*A*B by the 4M method (four real products, never
 * 3M) with the reference's alpha/beta special cases. alpha and beta are
 * (re, im) pairs. ComplexKernels.Multiply (src/Tensile/ComplexKernels.cs:49-108,
 * Combine :213-240); Workspace.Multiply(Complex) (src/Tensile/Workspace.Complex.cs:37-62). */
int tns_zgemm(tns_context* ctx, int m, int n, int k, const double* alpha, const double* a, int lda,
              const double* b, int ldb, const double* beta, double* c, int ldc);
int tns_zgemm_device(tns_context* ctx, int m, int n, int k, const double* alpha, const double* a,
                     int lda, const double* b, int ldb, const double* beta, double* c, int ldc);

/* ---- split-precision form ------------------------------------------------ */

/* C := A*B in the split-precision form: the rows of A and the columns of B
 * are scaled by powers of two and rounded to t-bit integers, their residues
 * modulo `moduli` (8..22) pairwise coprime moduli <= 256 are multiplied on the
 * 8-bit tensor cores with exact 32-bit accumulation, and the integer product
 * is rebuilt by the Chinese remainder theorem in FP64 (t is the largest with
 * 2 K 2^(2t) below the product of the moduli: 71 for 20 moduli and K <= 2048,
 * complex K counted twice). Each entry agrees with the exact product to about
 * K 2^-t of its row and column scales; it does not reproduce the reference's
 * rounding. Complex operands keep four real multiplications per complex
 * multiply-add (never 3M). No counterpart in the reference: this is the
 * split-precision form of ComplexKernels.Multiply
 * (src/Tensile/ComplexKernels.cs:49-108) and Gemm (src/Tensile.Kernels/Gemm.cs:117-203). */
int tns_dgemm_split(tns_context* ctx, int m, int n, int k, const double* a, int lda, const double* b, int ldb,
                    double* c, int ldc, int moduli);
int tns_zgemm_split(tns_context* ctx, int m, int n, int k, const double* a, int lda, const double* b, int ldb,
                    double* c, int ldc, int moduli);
/* 0 (the default): every product of Expm in plain FP64, the reference's
 * rounding. 8..22: Expm's products in the split-precision form with that
 * many moduli. The degree and s remain the reference's: the norm estimates
 * that select them stay in plain FP64, and d4, d6 come from A^4, A^6 in the
 * split form with bounds that hold the reference's values (its FP64
 * rounding included); a matrix whose decision is not settled on those
 * bounds has its A^2, A^4, A^6 recomputed as the reference computes them.
 * The LU and the solve of the Pade denominator keep the reference's
 * arithmetic. */
int tns_set_split_moduli(tns_context* ctx, int moduli);
/* 1: the GEMMs' launch shapes (the DMMA GEMM's small or big tiles, the
 * modular GEMM's 128- or 256-column tiles) are chosen by timing both on the
 * first launch of each size class (product kind, log2 of its tiles, log2 of its
 * depth) and remembered per device for the process; the shapes give identical
 * results, so only speed depends on the choice. A timed first launch of a
 * class waits for the stream. 0 (the default): big tiles when they fill the
 * GPU. No counterpart in the reference (its CPU blocking is fixed). */
int tns_set_autotune(tns_context* ctx, int enabled);

/* ---- exact norms -------------------------------------------------------- */

/* kind: '1' (largest column sum), 'I' (largest row sum), 'F' (Frobenius,
 * unscaled). Norms.One/Infinity/Frobenius (src/Tensile.Kernels/Norms.cs:11-66);
 * complex: ComplexKernels.OneNorm/InfinityNorm (src/Tensile/ComplexKernels.cs:144-180),
 * moduli by Complex.Abs. */
int tns_dnorm(tns_context* ctx, char kind, int m, int n, const double* a, int lda, double* out);
int tns_znorm(tns_context* ctx, char kind, int m, int n, const double* a, int lda, double* out);

/* ---- LU with partial pivoting ------------------------------------------- */

typedef struct {
    int singular_column;   /* first column with an exactly zero pivot, or -1 */
    double smallest_pivot; /* min |u_jj| (LuFactorization.SmallestPivot) */
    double largest_pivot;  /* max |u_jj| */
    double one_norm;       /* ||A||_1 of the input, captured before factoring */
} tns_lu_info;

/* In-place P*A = L*U (LAPACK packed form). pivots: min(m,n) 0-based entries,
 * row k swapped with pivots[k] in increasing k. nb <= 0 selects the reference
 * default (32 below min(m,n)=1024, else 64). Pivot rule: largest |a| (real) or
 * |Re|+|Im| (complex), ties to the lowest index.
 * Lu.Factor (src/Tensile.Kernels/Lu.cs:230-309) via KernelEntry.FactorLu
 * (src/Tensile.Kernels/KernelEntry.cs:59-67); complex BlockedLu.Factor
 * (src/Tensile/BlockedLu.cs:45-101) via Workspace.FactorLu(Complex)
 * (src/Tensile/Workspace.Complex.cs:79-104). */
int tns_dgetrf(tns_context* ctx, int m, int n, double* a, int lda, int nb, int* pivots,
               tns_lu_info* info);
int tns_zgetrf(tns_context* ctx, int m, int n, double* a, int lda, int nb, int* pivots,
               tns_lu_info* info);

/* Solve A X = B (adjoint = 0) or A^H X = B (adjoint = 1) in place from a
 * factorization; TNS_E_SINGULAR when singular_column >= 0.
 * Lu.Solve/SolveTransposed (src/Tensile.Kernels/Lu.cs:336-378) via
 * KernelEntry.SolveLu/SolveLuTransposed (src/Tensile.Kernels/KernelEntry.cs:70-95);
 * complex BlockedLu.Solve/SolveAdjoint (src/Tensile/BlockedLu.cs:105-141). */
int tns_dgetrs(tns_context* ctx, int n, int nrhs, const double* lu, int lda, const int* pivots,
               int singular_column, double* b, int ldb, int adjoint);
int tns_zgetrs(tns_context* ctx, int n, int nrhs, const double* lu, int lda, const int* pivots,
               int singular_column, double* b, int ldb, int adjoint);

/* The triangular solves of the kernel seam, in place: B := T^-1 B (or
 * T^-T B) for the m x m triangle T of A that the name gives (the other part of
 * A is not read), B m x n, in the reference's order of operations (column
 * axpys for the untransposed solves, ColumnOps.Dot inner products for the
 * transposed ones), so the result is the reference's bit for bit. A zero on
 * the diagonal divides by zero as the reference does (no error).
 * KernelEntry.SolveUpper, SolveUpperTransposed, SolveLower,
 * SolveLowerTransposed, SolveLowerUnit, SolveLowerUnitTransposed
 * (src/Tensile.Kernels/KernelEntry.cs:98-173; src/Tensile.Kernels/Triangular.cs:26-206),
 * as Structures.cs's UpperTriangular / LowerTriangular / UnitLowerTriangular
 * call them (src/Tensile/Structures.cs:96-167). */
int tns_dsolve_upper(tns_context* ctx, int m, int n, const double* a, int lda, double* b, int ldb);
int tns_dsolve_upper_transposed(tns_context* ctx, int m, int n, const double* a, int lda, double* b, int ldb);
int tns_dsolve_lower(tns_context* ctx, int m, int n, const double* a, int lda, double* b, int ldb);
int tns_dsolve_lower_transposed(tns_context* ctx, int m, int n, const double* a, int lda, double* b, int ldb);
int tns_dsolve_lower_unit(tns_context* ctx, int m, int n, const double* a, int lda, double* b, int ldb);
int tns_dsolve_lower_unit_transposed(tns_context* ctx, int m, int n, const double* a, int lda, double* b, int ldb);
/* The complex triangular solves the reference runs above its seam, in their
 * order of operations: BlockedLu.SolveUpper, SolveUpperAdjoint (U^H),
 * SolveLowerUnit, SolveLowerUnitAdjoint (L^H) (src/Tensile/BlockedLu.cs:283-373). */
int tns_zsolve_upper(tns_context* ctx, int m, int n, const double* a, int lda, double* b, int ldb);
int tns_zsolve_upper_adjoint(tns_context* ctx, int m, int n, const double* a, int lda, double* b, int ldb);
int tns_zsolve_lower_unit(tns_context* ctx, int m, int n, const double* a, int lda, double* b, int ldb);
int tns_zsolve_lower_unit_adjoint(tns_context* ctx, int m, int n, const double* a, int lda, double* b, int ldb);

/* Y := A X or Y := A^T X for square A (n x n) and panels X, Y (n x t).
 * KernelEntry.MultiplyPanel / MultiplyPanelTransposed
 * (src/Tensile.Kernels/KernelEntry.cs:176-201; PanelProduct.Apply /
 * ApplyTranspose, src/Tensile.Kernels/PanelProduct.cs:25-55), in their order
 * of operations. Complex: Y := A X or A^H X, ComplexDenseOperator.Apply /
 * ApplyAdjoint (src/Tensile/LinearOperators.cs:194-293). */
int tns_dmultiply_panel(tns_context* ctx, int n, int t, const double* a, int lda, const double* x, int ldx, double* y,
                        int ldy);
int tns_dmultiply_panel_transposed(tns_context* ctx, int n, int t, const double* a, int lda, const double* x, int ldx,
                                   double* y, int ldy);
int tns_zmultiply_panel(tns_context* ctx, int n, int t, const double* a, int lda, const double* x, int ldx, double* y,
                        int ldy);
int tns_zmultiply_panel_adjoint(tns_context* ctx, int n, int t, const double* a, int lda, const double* x, int ldx,
                                double* y, int ldy);

/* rcond = 1/(||A||_1 * est ||A^-1||_1), 0 when singular or ||A||_1 == 0.
 * Condition.ReciprocalOne (src/Tensile/NormEstimate.cs:432-466) over
 * LuInverseOperator (src/Tensile/LinearOperators.cs:303-350). */
int tns_dgecon(tns_context* ctx, int n, const double* lu, int lda, const int* pivots,
               int singular_column, double anorm, double* rcond);
int tns_zgecon(tns_context* ctx, int n, const double* lu, int lda, const int* pivots,
               int singular_column, double anorm, double* rcond);

/* ---- block 1-norm estimation -------------------------------------------- */

typedef struct {
    double value;   /* lower bound on ||A^power||_1 */
    int iterations;
    int products;   /* operator applications, counting each probe column */
} tns_normest_result;

/* NormEstimate.Estimate (src/Tensile/NormEstimate.cs:104-274) over the dense
 * power operators DenseMatrixOperator / ComplexDenseOperator
 * (src/Tensile/LinearOperators.cs:89-293). t, itmax and seed as
 * NormEstimate.Of (defaults 2, 5, 20260915). */
int tns_dnormest1_power(tns_context* ctx, int n, const double* a, int lda, int power, int t, int itmax,
                        int seed, tns_normest_result* out);
int tns_znormest1_power(tns_context* ctx, int n, const double* a, int lda, int power, int t, int itmax,
                        int seed, tns_normest_result* out);

/* ---- matrix exponential ------------------------------------------------- */

typedef struct {
    int degree;    /* Pade degree 3, 5, 7, 9 or 13; 0 for n <= 1 */
    int squarings; /* s */
} tns_expm_info;

/* exp(A) by Al-Mohy & Higham 2009 scaling and squaring.
 * MatrixExponential.Expm (src/Tensile/MatrixExponential.cs:136-270;
 * complex src/Tensile/MatrixExponential.Complex.cs:35-53); info mirrors
 * ExpmDiagnostics (:575-582). TNS_E_SINGULAR: singular Pade denominator. */
int tns_dexpm(tns_context* ctx, int n, const double* a, int lda, double* out, int ldo, tns_expm_info* info);
int tns_zexpm(tns_context* ctx, int n, const double* a, int lda, double* out, int ldo, tns_expm_info* info);

/* A batch of complex exponentials of independent orders: out[i] = exp(a[i]).
 * The frequency-sweep form of the same algorithm; every decision per matrix
 * is the one tns_zexpm takes. Host pointers (synchronous) or, for
 * _device, device pointers. infos may be NULL. With page-locked host outputs
 * each result is copied out as soon as it is final, while the other matrices
 * are still being computed; pageable outputs are copied at the end. */
int tns_zexpm_batched(tns_context* ctx, int count, const int* orders, const double* const* a,
                      const int* lda, double* const* out, const int* ldo, tns_expm_info* infos);
int tns_zexpm_batched_device(tns_context* ctx, int count, const int* orders, const double* const* a,
                             const int* lda, double* const* out, const int* ldo, tns_expm_info* infos);
/* How many groups a batch is split into. Each group (cost-balanced, n^3 as the
 * cost) runs the batched algorithm -- one launch per phase for all its
 * matrices -- on its own host thread and CUDA stream. Default 4. */
int tns_set_workers(tns_context* ctx, int workers);

/* ---- action of the exponential ------------------------------------------ */

typedef struct {
    int degree;       /* Taylor degree m (a cap) */
    int scaling;      /* s >= 1 */
    int applications; /* operator applications performed */
    int early_exits;  /* inner loops stopped by the tolerance test */
} tns_expmv_info;

/* exp(tA)B for dense A (trace shift, sharp ||A^p||^(1/p) bounds, early exit).
 * MatrixExponentialAction.Expmv (src/Tensile/MatrixExponentialAction.cs:113-320;
 * complex src/Tensile/MatrixExponentialAction.Complex.cs:34-63); info mirrors
 * ExpmvDiagnostics (:498-511). TNS_E_OUT_OF_RANGE when the application count
 * cannot be represented (:386-395). */
int tns_dexpmv(tns_context* ctx, int n, const double* a, int lda, int ncols, const double* b, int ldb,
               double t, double* out, int ldo, tns_expmv_info* info);
int tns_zexpmv(tns_context* ctx, int n, const double* a, int lda, int ncols, const double* b, int ldb,
               double t, double* out, int ldo, tns_expmv_info* info);

/* A batch of exponential actions out[i] = exp(t a[i]) b[i] of independent
 * orders (every b[i] with ncols columns): the frequency-sweep form of
 * tns_dexpmv / tns_zexpmv, each matrix with the reference's trace shift,
 * sharp bounds, (m, s) and early exit. The parameters of all matrices are
 * chosen together (their normest1 runs advanced in lockstep); the Taylor
 * recurrences of all of them then run in one cooperative kernel launch, the
 * early-exit test on the device. Each result is the reference's arithmetic
 * (MatrixExponentialAction.Run, src/Tensile/MatrixExponentialAction.cs:239-320),
 * so it equals tns_zexpmv on the same matrix bit for bit. Orders may be 0
 * (nothing is written). infos may be NULL. _device: device pointers. */
int tns_dexpmv_batched(tns_context* ctx, int count, const int* orders, const double* const* a, const int* lda,
                       int ncols, const double* const* b, const int* ldb, double t, double* const* out,
                       const int* ldo, tns_expmv_info* infos);
int tns_zexpmv_batched(tns_context* ctx, int count, const int* orders, const double* const* a, const int* lda,
                       int ncols, const double* const* b, const int* ldb, double t, double* const* out,
                       const int* ldo, tns_expmv_info* infos);
int tns_zexpmv_batched_device(tns_context* ctx, int count, const int* orders, const double* const* a,
                              const int* lda, int ncols, const double* const* b, const int* ldb, double t,
                              double* const* out, const int* ldo, tns_expmv_info* infos);

/* Only the (m, s) that tns_zexpmv_batched would choose for each complex
 * matrix, with panels of ncols columns and this t (trace shift, sharp
 * bounds, the search of MatrixExponentialAction.SelectParameters,
 * src/Tensile/MatrixExponentialAction.cs:347-398), without running the
 * recurrences: infos[i].degree and .scaling; applications and early_exits
 * stay 0. Lets a caller see the cost (m s applications) of a sweep before
 * running it. _device: device pointers. */
int tns_zexpmv_select_batched(tns_context* ctx, int count, const int* orders, const double* const* a, const int* lda,
                              int ncols, double t, tns_expmv_info* infos);
int tns_zexpmv_select_batched_device(tns_context* ctx, int count, const int* orders, const double* const* a,
                                     const int* lda, int ncols, double t, tns_expmv_info* infos);

/* ---- precision form of the solve ----------------------------------------- */

typedef struct {
    int moduli;            /* moduli of the factorization the refinement used */
    int factorizations;    /* 1, or 2 when the condition estimate asked for more precision */
    int iterations;        /* refinement steps taken */
    double backward_error; /* max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf) at the end */
    double rcond;          /* 1 / (||A||_1 est ||A^-1||_1) through the factors the refinement used */
    int pivoting;          /* 0: butterfly transforms, no row interchanges; 1: partial pivoting ran */
} tns_mixed_info;

/* X := A^-1 B (A n x n, B and X n x nrhs) by a low-precision LU and FP64
 * iterative refinement. The LU's trailing updates (depth 512), nearly all of
 * its flops, run on the split-precision product with `moduli` moduli (8..22;
 * the integer images keep 26 bits with 8, 49 with 14); panels of 512 columns
 * are factored in FP64. First route: A becomes T A S with random butterfly
 * transforms (depth 2, order padded to a multiple of 4) and is factored
 * without row interchanges; if that meets an exactly zero pivot or its
 * refinement ends above 8 u, the solve runs again with partial pivoting
 * (info->pivoting = 1, info->factorizations counting both routes). The
 * refinement computes residuals with A itself in FP64 and stops when the
 * backward error reaches 4 u, stops halving, or after max_iter steps.
 * moduli = 0: chosen from the condition estimate kappa_1 of a first 8-moduli
 * factorization so that the images keep log2(kappa_1) + 7 bits (refactoring
 * once when that needs more). No counterpart in the reference, whose solve
 * (Lu.Factor + Lu.Solve, src/Tensile.Kernels/Lu.cs:230-351) is FP64 throughout;
 * this is its precision form. TNS_E_SINGULAR for an exactly zero pivot. */
int tns_dgesv_mixed(tns_context* ctx, int n, int nrhs, const double* a, int lda, const double* b, int ldb, double* x,
                    int ldx, int moduli, int max_iter, tns_mixed_info* info);
int tns_zgesv_mixed(tns_context* ctx, int n, int nrhs, const double* a, int lda, const double* b, int ldb, double* x,
                    int ldx, int moduli, int max_iter, tns_mixed_info* info);

/* ---- differentiation: Frechet derivative and adjoint ---------------------- */

/* exp(A) and its Frechet derivative L(A, E) = d/dh exp(A + hE) at h = 0, both
 * n x n. No counterpart in the reference: Tensile obtains L(A, E) only as the
 * upper right block of its Expm of the 2n x 2n matrix [[A, E], [0, A]]
 * (MatrixExponential.ScalingAndSquaring, src/Tensile/MatrixExponential.cs:181-270);
 * this computes the same quantity at about three times the cost of one Expm
 * (Al-Mohy and Higham 2009, Algorithm 6.4). expa may be NULL (then ldx is not
 * read). info (may be NULL) receives the Pade degree and the squarings of that
 * algorithm, not the reference's Expm decisions. TNS_E_ARGUMENT for a
 * non-finite A. */
int tns_dexpm_frechet(tns_context* ctx, int n, const double* a, int lda, const double* e, int lde, double* expa,
                      int ldx, double* l, int ldl, tns_expm_info* info);
int tns_zexpm_frechet(tns_context* ctx, int n, const double* a, int lda, const double* e, int lde, double* expa,
                      int ldx, double* l, int ldl, tns_expm_info* info);

/* The gradient of loss = ||exp(tA) B - Y||_F^2 (A n x n, B and Y n x ncols):
 * loss, and dloss/dA (n x n), dloss/dB (n x ncols), dloss/dt, with
 * dloss = Re <grad, d.> and <X, Y> = trace(X^H Y), so that a complex gradient
 * holds the derivatives with respect to the real and imaginary parts. f (may
 * be NULL) receives exp(tA) B. No counterpart in the reference: it is the
 * adjoint of MatrixExponentialAction.Expmv
 * (src/Tensile/MatrixExponentialAction.cs:113-142), computed from one forward
 * pass of the Frechet algorithm on t A^H and one derivative pass in the
 * direction G B^H, G = 2 (exp(tA) B - Y). */
int tns_dexpmv_gradient(tns_context* ctx, int n, int ncols, double t, const double* a, int lda, const double* b,
                        int ldb, const double* y, int ldy, double* loss, double* grad_a, int ldga, double* grad_b,
                        int ldgb, double* grad_t, double* f, int ldf, tns_expm_info* info);
int tns_zexpmv_gradient(tns_context* ctx, int n, int ncols, double t, const double* a, int lda, const double* b,
                        int ldb, const double* y, int ldy, double* loss, double* grad_a, int ldga, double* grad_b,
                        int ldgb, double* grad_t, double* f, int ldf, tns_expm_info* info);

/* Device bytes the Frechet derivative may hold for the squarings of its
 * forward pass. Within the budget every squaring is kept for the derivative
 * pass; beyond it only the first is, and the derivative pass squares again
 * (more products, less memory). -1 (the default): a quarter of the free
 * device memory at the time of the call. */
int tns_set_checkpoint_bytes(tns_context* ctx, long long bytes);

/* ---- matrix-free exponential action ------------------------------------- */

/* A matrix-free operator: the device-side ILinearOperator<T>.Apply
 * (src/Tensile/LinearOperators.cs:37-75). It must write y := A x for the
 * n x ncols panel x. Both panels are in device memory, column-major with
 * leading dimension ld in elements (complex: interleaved (re, im) pairs).
 * The work goes on `stream` (a cudaStream_t, the context's stream), in stream
 * order; the callback may launch its own kernels there. It returns 0 on
 * success; any other value ends the call with TNS_E_OPERATOR. The panels
 * stay on the device from one application to the next: no host copy per
 * application. */
typedef int (*tns_apply_fn)(void* user, int ncols, const double* x, double* y, int ld, void* stream);

/* exp(tA)B for an operator known only through `apply`
 * (MatrixExponentialAction.Expmv(ILinearOperator<T>, B, t, oneNormBound),
 * src/Tensile/MatrixExponentialAction.cs:203-230; complex .Complex.cs:85-111).
 * The reference's semantics: no trace shift (mu = 0), one_norm_bound an upper
 * bound on ||A||_1 (finite, >= 0, else TNS_E_OUT_OF_RANGE), and the degree and
 * scaling from the crude bound |t| one_norm_bound alone, with no norm
 * estimation, so (m, s) are the reference's exactly. apply NULL:
 * TNS_E_NULL. */
int tns_dexpmv_operator(tns_context* ctx, int n, tns_apply_fn apply, void* user, int ncols, const double* b, int ldb,
                        double t, double one_norm_bound, double* out, int ldo, tns_expmv_info* info);
int tns_zexpmv_operator(tns_context* ctx, int n, tns_apply_fn apply, void* user, int ncols, const double* b, int ldb,
                        double t, double one_norm_bound, double* out, int ldo, tns_expmv_info* info);

/* NormEstimate.Of(IAdjointOperator<T>, columns, maxIterations, seed)
 * (src/Tensile/NormEstimate.cs:70-93, the estimator :104-274) for a caller's
 * operator: `apply` writes y := A x and `adjoint` writes y := A^H x, both as
 * tns_apply_fn on device panels (n x t). The estimator's bookkeeping is the
 * reference's. When the operator's products are exact, the estimate, iteration
 * count and product count equal the reference's exactly. apply or adjoint
 * NULL: TNS_E_NULL; a callback's failure: TNS_E_OPERATOR. */
int tns_dnormest1_operator(tns_context* ctx, int n, tns_apply_fn apply, tns_apply_fn adjoint, void* user, int t,
                           int itmax, int seed, tns_normest_result* out);
int tns_znormest1_operator(tns_context* ctx, int n, tns_apply_fn apply, tns_apply_fn adjoint, void* user, int t,
                           int itmax, int seed, tns_normest_result* out);

/* ---- complex product without allocation -------------------------------- */

/* No counterpart in the reference: the reference's products run on the CPU
 * with managed buffers and have no device memory to avoid.
 *
 * C := beta*C + alpha*A*B for complex device operands, the same 4M product and
 * the same bits as tns_zgemm_device, for callers that may not allocate device
 * memory when they need the product -- for instance a host application whose
 * own allocator has reserved the GPU's memory up front, or a latency-critical
 * loop that must not enter the driver's allocation path. It allocates nothing:
 * its working storage is one fixed device array of 4,194,304 complex elements
 * (64 MiB) inside the library, which every GPU that loads the library holds
 * until the process exits. A product whose padded operands need more than that
 * (roughly m*k + k*n + 2*m*n complex elements, with m rounded up to even and k
 * to a multiple of 16) is refused with TNS_E_OUT_OF_RANGE; tns_last_error(NULL)
 * says why. There is no context: stream is the caller's cudaStream_t (NULL for
 * the default stream) on the current device. Every call waits for that stream
 * before it returns: it reads the product kernel's wait flag first and copies
 * the product into C only when no device-side wait gave up (TNS_E_TIMEOUT
 * leaves C untouched). k == 0 scales C by beta and reads neither alpha nor
 * the working array, as tns_zgemm_device does.
 *
 * The first call on a device looks up the array's device address, with that
 * device current; make that first call before any stream capture. All calls
 * share the array, which keeps the previous call's contents; calls that
 * overlap on the GPU (from several threads or streams) race on it. */
int tns_zgemm_device_noalloc(void* stream, int m, int n, int k, const double* alpha, const double* a, int lda,
                             const double* b, int ldb, const double* beta, double* c, int ldc);

/* ---- diagnostics --------------------------------------------------------- */

/* Counters of the work a context has issued, the device-side counterpart of
 * the reference's LuPhaseTimings / ExpmDiagnostics observers
 * (src/Tensile.Kernels/Lu.cs:92-164, src/Tensile/MatrixExponential.cs:575-582).
 * gemm_ms is the summed CUDA-event duration of the GEMM kernel launches made
 * while timing was enabled; gemm_flops counts 2mnk (real) or 8mnk (complex 4M)
 * at the products' true sizes; gemm_bytes is the least memory traffic of
 * those launches (A and B read once, C written once and read once when beta
 * is non-zero) at the launched sizes (m, n rounded up to even, k to a multiple
 * of 16). */
typedef struct {
    long long kernel_launches; /* every kernel this context launched */
    long long gemm_launches;
    double gemm_flops;
    double gemm_ms;
    double gemm_bytes;
    /* the split-precision product's launches: FP64-equivalent flops (8mnk /
     * 2mnk), 8-bit tensor operations actually issued, and their event time */
    long long split_launches;
    double split_flops;
    double split_int8_ops;
    double split_ms;
    /* algorithmic bytes of the modular GEMM launches: every modulus' 8-bit
     * residue images of A and B read once and its 8-bit result plane written
     * once, at the padded extents */
    double split_bytes;
    /* size classes the autotuner timed (tns_set_autotune) */
    long long autotune_trials;
    /* split form: matrices whose A^2, A^4, A^6 were recomputed in plain FP64
     * because a degree or s decision was not settled on the split values */
    long long exact_fallbacks;
} tns_stats;

int tns_get_stats(tns_context* ctx, tns_stats* out); /* waits for the stream */

/* LuPhaseTimings (src/Tensile.Kernels/Lu.cs:92-164) on the device: with
 * collection switched on, every blocked LU this context runs (tns_dgetrf,
 * tns_zgetrf and the factorizations inside the solves and exponentials it
 * runs itself) records CUDA events between its phases -- the panel
 * factorization, the row interchanges, the triangular solve for U12, the
 * trailing GEMM -- and around the whole blocked loop. A timed factorization
 * waits for its stream once at the end. A factorization that is one
 * whole-matrix panel has no blocked loop and records nothing, as in the
 * reference. unattributed_ms is total_ms minus the phases, never negative
 * (LuPhaseTimings.Unattributed). tns_reset_stats clears the sums. */
typedef struct {
    double panel_ms, swaps_ms, triangular_ms, gemm_ms, total_ms, unattributed_ms;
    long long block_steps, factorizations;
} tns_lu_timings;
int tns_set_lu_timing(tns_context* ctx, int enabled);
int tns_get_lu_timings(tns_context* ctx, tns_lu_timings* out);
int tns_reset_stats(tns_context* ctx);
int tns_set_timing(tns_context* ctx, int enabled);
/* Failure paths, exercised without a GPU fault. The k-th device allocation
 * this context makes from now (counting the padded operand copies and work
 * matrices of every call) fails as a cudaMalloc that ran out of memory would:
 * the call returns TNS_E_OUT_OF_MEMORY with its destination untouched, and
 * the next allocation succeeds again. k = 0 disarms it. No counterpart in the
 * reference (its managed allocations throw OutOfMemoryException). */
int tns_inject_allocation_failure(tns_context* ctx, long long k);
/* Runs one kernel whose bounded wait, on a barrier that nothing arrives on,
 * gives up after limit_ns nanoseconds (at most 2e9), as every device-side
 * wait of the library does after its own limit: the call returns TNS_E_TIMEOUT
 * and the context stays usable. */
int tns_selftest_wait(tns_context* ctx, long long limit_ns);

/* The CUDA stream (cudaStream_t) the context issues its work on. */
int tns_get_stream(tns_context* ctx, void** stream);

#ifdef __cplusplus
}
#endif
#endif
