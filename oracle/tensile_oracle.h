/*
 * CPU oracle for the Tensile dense hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A C++ restatement of the reference library's CPU algorithms (the managed C#
 * Tensile library, xfmrexpert/CSharp_LinearAlgebra). It exists to check the
 * CUDA library and to serve as the timed CPU baseline. Nothing in the product
 * path (csharp_linearalgebra_b200/) may call it.
 *
 * Parity status: PARTIALLY PINNED. The reference cannot be executed here (it
 * is .NET 10 managed code and no .NET runtime exists on either machine), so
 * the restatement is pinned by the reference's own known-answer tests (Pade
 * coefficients, closed-form exponentials, pivot rules, every Pade degree
 * reached on the reference's seeded inputs, estimator invariants) and by
 * independent cross-checks against scipy. Bit patterns of .NET's seeded
 * System.Random and Array.Sort are restated from their published algorithms
 * and are unverifiable without a .NET runtime.
 *
 * All matrices are column-major with a leading dimension; complex values are
 * interleaved (re, im) pairs of doubles, the layout of System.Numerics.Complex.
 */
#ifndef TENSILE_ORACLE_H
#define TENSILE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- .NET System.Random(int seed) legacy subtractive generator ---------- */
typedef struct orc_random orc_random;
orc_random* orc_random_new(int seed);
void orc_random_free(orc_random* r);
int orc_random_next(orc_random* r, int max_value);   /* Random.Next(max) */
double orc_random_next_double(orc_random* r);        /* Random.NextDouble() */

/* .NET Array.Sort(double[] keys, int[] items): introsort, NaN prepass. */
void orc_sort_keys_items(int n, double* keys, int* items);

/* ---- GEMM: C := beta*C + alpha*A*B ------------------------------------- */
/* threads <= 0: all cores. multithreaded selects the reference's threaded
 * dispatch (KC=256 at and above 2^24 work, else the serial KC=384). */
void orc_set_threads(int threads);
int orc_get_threads(void);
int orc_dgemm(int m, int n, int k, double alpha, const double* a, int lda,
              const double* b, int ldb, double beta, double* c, int ldc, int multithreaded);
int orc_zgemm(int m, int n, int k, const double* alpha, const double* a, int lda,
              const double* b, int ldb, const double* beta, double* c, int ldc, int multithreaded);

/* ---- norms --------------------------------------------------------------- */
double orc_dnorm1(int m, int n, const double* a, int lda);
double orc_dnorminf(int m, int n, const double* a, int lda);
double orc_dnormfro(int m, int n, const double* a, int lda);
double orc_znorm1(int m, int n, const double* a, int lda);
double orc_znorminf(int m, int n, const double* a, int lda);
double orc_zabs(double re, double im); /* Complex.Abs */

/* ---- LU with partial pivoting (in place) -------------------------------- */
typedef struct {
    int singular_column;   /* -1 when every pivot is non-zero */
    double smallest_pivot; /* min |u_jj| */
    double largest_pivot;  /* max |u_jj| */
} orc_lu_info;

int orc_dgetrf(int m, int n, double* a, int lda, int nb, int* pivots, orc_lu_info* info);
int orc_zgetrf(int m, int n, double* a, int lda, int nb, int* pivots, orc_lu_info* info);
/* adjoint=0: A X = B; adjoint=1: A^H X = B. Returns 2 when singular. */
int orc_dgetrs(int n, int nrhs, const double* lu, int lda, const int* pivots, int singular_column,
               double* b, int ldb, int adjoint);
int orc_zgetrs(int n, int nrhs, const double* lu, int lda, const int* pivots, int singular_column,
               double* b, int ldb, int adjoint);

/* Triangular solves of the kernel seam, in place: kind 0 upper, 1 upper^T,
 * 2 lower, 3 lower^T, 4 unit lower, 5 unit lower^T (Triangular.cs); complex
 * (BlockedLu's generic solves): 0 upper, 1 upper^H, 4 unit lower, 5 unit
 * lower^H. Returns 1 for an unknown kind. */
int orc_dtrsolve(int kind, int m, int n, const double* a, int lda, double* b, int ldb);
int orc_ztrsolve(int kind, int m, int n, const double* a, int lda, double* b, int ldb);
/* Y := A X or A^T X (PanelProduct); complex: the dense operator's A X / A^H X. */
int orc_dpanel(int transposed, int n, int t, const double* a, int lda, const double* x, int ldx, double* y, int ldy);
int orc_zpanel(int adjoint, int n, int t, const double* a, int lda, const double* x, int ldx, double* y, int ldy);

/* ---- Higham-Tisseur block 1-norm estimator ------------------------------ */
typedef struct {
    double value;
    int iterations;
    int products;
} orc_normest_result;

/* ||A^p||_1 for a dense square matrix, never forming A^p. */
int orc_dnormest_power(int n, const double* a, int lda, int power, int t, int itmax, int seed,
                       orc_normest_result* out);
int orc_znormest_power(int n, const double* a, int lda, int power, int t, int itmax, int seed,
                       orc_normest_result* out);
/* Reciprocal 1-norm condition number from an LU factorization. */
int orc_dgecon(int n, const double* lu, int lda, const int* pivots, int singular_column,
               double anorm, double* rcond);
int orc_zgecon(int n, const double* lu, int lda, const int* pivots, int singular_column,
               double anorm, double* rcond);

/* ---- matrix exponential and its action ---------------------------------- */
typedef struct {
    int degree;
    int squarings;
    /* decision inputs, reported so that a tie can be told from a mismatch */
    double eta1, eta3, eta5, d4, d6, d8, d10;
} orc_expm_info;

typedef struct {
    int degree;
    int scaling;
    int applications;
    int early_exits;
} orc_expmv_info;

int orc_dexpm(int n, const double* a, int lda, double* out, int ldo, orc_expm_info* info);
int orc_zexpm(int n, const double* a, int lda, double* out, int ldo, orc_expm_info* info);
/* Matrix-free Expmv: mu = 0, the caller's bound on ||A||_1, no estimator
 * (MatrixExponentialAction.cs:203-230, .Complex.cs:85-111); A applied densely. */
int orc_dexpmv_bound(int n, const double* a, int lda, int ncols, const double* b, int ldb, double t, double bound,
                     double* out, int ldo, orc_expmv_info* info);
int orc_zexpmv_bound(int n, const double* a, int lda, int ncols, const double* b, int ldb, double t, double bound,
                     double* out, int ldo, orc_expmv_info* info);
int orc_dexpmv(int n, const double* a, int lda, int ncols, const double* b, int ldb, double t,
               double* out, int ldo, orc_expmv_info* info);
int orc_zexpmv(int n, const double* a, int lda, int ncols, const double* b, int ldb, double t,
               double* out, int ldo, orc_expmv_info* info);
/* The (m, s) Expmv selects (trace shift, sharp bounds, the search) without
 * running the Taylor recurrence; applications stay 0. */
int orc_dexpmv_params(int n, const double* a, int lda, int ncols, double t, orc_expmv_info* info);
int orc_zexpmv_params(int n, const double* a, int lda, int ncols, double t, orc_expmv_info* info);

#ifdef __cplusplus
}
#endif
#endif
