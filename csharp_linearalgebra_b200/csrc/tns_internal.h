// Internal host-side interfaces of the tensile_b200 library: the context
// (one CUDA stream per workspace), error handling, padded device matrices and
// the launchers of the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tensile_b200.h"

namespace tns {

// Thrown inside the library, caught at the C ABI and mapped to a status code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const std::string& msg);
[[noreturn]] void fail_cuda(cudaError_t e, const char* what, const char* file, int line);

#define TNS_CUDA(x)                                                  \
    do {                                                             \
        cudaError_t e_ = (x);                                        \
        if (e_ != cudaSuccess) ::tns::fail_cuda(e_, #x, __FILE__, __LINE__); \
    } while (0)

// Device matrices are zero-padded to multiples of this many rows and columns,
// which makes every GEMM operand meet the bulk-copy alignment rules and lets
// the LU and solves work on whole 64-wide blocks.
constexpr int kPad = 64;
inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// One problem of a (grouped) GEMM: C := beta*C + alpha*A*B. lda/ldb/ldc are in
// elements (complex elements for complex problems).
//
// kc is the reference's KC slab depth (Gemm.cs / ParallelGemm.cs): the
// accumulator is folded into C as c = fma(alpha, acc, c) at the end of every
// kc-deep slab of K, exactly where the reference's micro-kernel writes back.
// 0 lets gemm() choose the reference's rule for the problem's true size.
// W (complex only): scratch for the 4M partial products P + iQ, M x N with
// leading dimension ldw; null when the result can be written straight into C.
struct GemmProblem {
    const void* A;
    const void* B;
    void* C;
    int lda, ldb, ldc;
    int M, N, K;
    int tiles_m, tiles_n, tile_begin;
    double alpha_re, alpha_im, beta_re, beta_im;
    int kc;
    void* W;
    int ldw;
    long long work;  // m*n*k of the unpadded product, for the KC rule
    // Slab-split launches only (one product whose tiles leave SMs idle): each
    // KC slab's raw product (per pass, complex) lands in its own M x N plane
    // of S, and a fold kernel adds the slabs into C in slab order.
    void* S;
    int slabs;
};

// The reference's KC rule (GemmDispatch.cs:45,109; Gemm.cs:62; ParallelGemm):
// the default multithreaded workspace runs products of at least 2^24 work
// threaded with KC = 256, smaller ones serially with KC = 384.
inline int reference_kc(long long work) { return work >= (1LL << 24) ? 256 : 384; }

struct Context {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    int* d_err = nullptr;           // device-side error flag (bounded waits)
    unsigned long long* d_tiles = nullptr;  // grouped GEMM's tile counter, zeroed before each launch
    long long max_elements = 2147483591LL;
    std::string last_error;
    long long kernel_launches = 0;  // kernels launched through this context
    // Launch descriptors go to the device through a ring of pinned host memory
    // mirrored in device memory, so that uploading them never blocks the host
    // on the stream. Wrapping around synchronises the stream once.
    char* h_ring = nullptr;
    char* d_ring = nullptr;
    size_t ring_cap = 0, ring_pos = 0;
    const void* upload(const void* src, size_t bytes);

    // Optional per-launch timing of the GEMM kernel (CUDA events on this
    // context's stream), for the roofline report.
    bool timing = false;
    long long gemm_launches = 0;
    double gemm_flops = 0.0;  // algorithmic: 2mnk real, 8mnk complex (4M), true sizes
    double gemm_bytes = 0.0;  // least traffic: A, B read, C written (and read if beta != 0)
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> gemm_events;
    std::vector<cudaEvent_t> event_pool;
    double gemm_ms_done = 0.0;  // elapsed time of events already drained
    // The split-precision product's launches (counted and timed apart from the
    // FP64 GEMM's): FP64-equivalent algorithmic flops and 8-bit operations.
    int split_moduli = 0;       // 0: Pade and squaring products in plain FP64
    // Device bytes the Frechet derivative may spend on keeping every squaring
    // of its forward pass (else it keeps X_0 and squares again); -1: a quarter
    // of the free device memory.
    long long checkpoint_bytes = -1;
    // Launch shapes of the GEMMs chosen by timing both on a size class's
    // first launch (autotune.h) instead of the fixed rule.
    bool autotune = false;
    long long autotune_trials = 0;
    // A batch worker: its kernels share the GPU with other workers' streams,
    // so it launches nothing that needs the whole GPU at once (the
    // cooperative LU panel).
    bool concurrent = false;
    // Split form: matrices whose A^2, A^4, A^6 were recomputed in plain FP64
    // because a decision was not settled on the split values' intervals.
    long long exact_fallbacks = 0;
    long long split_launches = 0;
    double split_flops = 0.0, split_int8_ops = 0.0, split_ms_done = 0.0, split_bytes = 0.0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> split_events;
    // The split product's residue planes (gigabytes for a batch) live in one
    // grow-only buffer reused in stream order, instead of passing through the
    // stream-ordered pool at every launch, where four streams' churn of such
    // blocks can force fresh mappings.
    void* split_scratch = nullptr;
    size_t split_scratch_bytes = 0;
    void* scratch(size_t bytes);
    cudaEvent_t take_event();
    void drain_events();        // sums finished event pairs into gemm_ms_done / split_ms_done

    // LuPhaseTimings' device counterpart (tns_set_lu_timing): CUDA-event time
    // of the blocked LU's phases, summed over the factorizations timed.
    bool lu_timing = false;
    double lu_panel_ms = 0.0, lu_swaps_ms = 0.0, lu_triangular_ms = 0.0, lu_gemm_ms = 0.0, lu_total_ms = 0.0;
    long long lu_block_steps = 0, lu_factorizations = 0;

    // A second stream for copies of finished results that overlap the work
    // still running on `stream` (created on first use).
    cudaStream_t copy_stream = nullptr;
    cudaStream_t copies();

    // Batched work runs on worker contexts (one host thread and one stream
    // each), created on first use, so that independent matrices overlap on
    // the GPU. Their counters are summed into this context's statistics.
    int max_workers = 4;
    std::vector<std::unique_ptr<Context>> workers;

    // Device allocations made through DMat, DBuf and the split scratch, and
    // the test hook that fails one of them (tns_inject_allocation_failure).
    long long allocations = 0;
    long long fail_allocation_at = 0;  // 0: off; else the allocation number that fails
    void count_allocation();

    explicit Context(int dev);
    ~Context();
    void sync();                       // stream sync + device error flag check
    void check_limit(long long elements, const char* purpose) const;
};

// A padded device matrix owned by the library: rows_p x cols_p with
// ld = rows_p, zero outside rows x cols. Freed on the context's stream.
struct DMat {
    Context* ctx = nullptr;
    double* p = nullptr;
    int rows = 0, cols = 0, rows_p = 0, cols_p = 0;
    bool cplx = false;

    DMat() = default;
    DMat(Context& c, int r, int k, bool complex_, const char* purpose = "a device matrix");
    DMat(const DMat&) = delete;
    DMat& operator=(const DMat&) = delete;
    DMat(DMat&& o) noexcept { *this = std::move(o); }
    DMat& operator=(DMat&& o) noexcept;
    ~DMat();
    int ld() const { return rows_p; }
    int esz() const { return cplx ? 16 : 8; }
    size_t bytes() const { return (size_t)rows_p * cols_p * esz(); }
    double* col(int j) { return p + (size_t)j * rows_p * (cplx ? 2 : 1); }
    double* at(int i, int j) { return p + ((size_t)j * rows_p + i) * (cplx ? 2 : 1); }
    const double* at(int i, int j) const { return p + ((size_t)j * rows_p + i) * (cplx ? 2 : 1); }
    void zero();
};

// Scoped device scratch on the context's stream.
struct DBuf {
    Context* ctx = nullptr;
    void* p = nullptr;
    size_t bytes = 0;
    DBuf() = default;
    DBuf(Context& c, size_t b);
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept { *this = std::move(o); }
    DBuf& operator=(DBuf&& o) noexcept;
    ~DBuf();
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// Launch a kernel whose bounded wait on a barrier nothing arrives on gives up
// after limit_ns and records the device error (the timeout path's self-test).
void selftest_wait(Context& ctx, long long limit_ns);

// ---- transfers -------------------------------------------------------------
// Copy a rows x cols column-major operand (host or device pointer, ld in
// elements) into / out of a padded device matrix.
void copy_in(Context& ctx, DMat& dst, const double* src, int ld, bool src_on_device);
void copy_out(Context& ctx, const DMat& src, double* dst, int ld, bool dst_on_device);
// The same on another stream (the caller orders it after the producer).
void copy_out_on(cudaStream_t stream, const DMat& src, double* dst, int ld, bool dst_on_device);
void copy_dmat(Context& ctx, DMat& dst, const DMat& src);

// ---- GEMM (gemm.cu) --------------------------------------------------------
void gemm_grouped(Context& ctx, std::vector<GemmProblem>& probs, bool cplx);
void gemm(Context& ctx, const GemmProblem& p, bool cplx);
GemmProblem make_gemm(const DMat& a, const DMat& b, DMat& c, double alpha_re, double alpha_im, double beta_re,
                      double beta_im);
// One complex product on a caller's stream, with no context: allocates and
// uploads nothing (the entry point for callers that cannot allocate).
void gemm_detached_complex(cudaStream_t stream, int device, int* d_err, const GemmProblem& p);
// Split-precision products C := A B (beta 0) or C += A B (beta 1) from
// 8-bit residues modulo `moduli` coprime moduli on the tcgen05 tensor cores,
// reconstructed by the Chinese remainder theorem (ozaki.cu).
struct SplitProduct {
    const DMat* a;
    const DMat* b;
    DMat* c;
    double beta;
};
void gemm_split_batch(Context& ctx, std::vector<SplitProduct>& v, int moduli);
// Integer bits t of the operands' images for `moduli` moduli and products of depth kmax.
int split_integer_bits(int moduli, int kmax);
// The thread's message for errors raised outside any context (tns_last_error(NULL)).
void set_detached_error(const std::string& msg);

// ---- batched streaming kernels (blas1.cu) ----------------------------------
// Descriptors of one item each; a batch of them runs in one launch.
struct EwDesc {
    int op;
    double* dst;
    double* dst2;
    const double* s1;
    const double* s2;
    size_t count;  // doubles
    double f;
    int rows_p, n, cplx;
};
struct SumDesc {  // moduli sums of an m x n block (or a fold of n values into out[0])
    const double* a;
    int m, n, ld;
    double* out;
};
struct ChainDesc {  // the ell test's abs-power chain of one matrix
    const double* a;
    int n, ld;
    double* mags;
    double* row;
    double* next;
};
struct PanelDesc {  // Y := A X (or A^H X), X and Y n x t
    const double* a;
    int n, ld;
    const double* x;
    int ldx;
    double* y;
    int ldy, t;
};
void ew_batch(Context& ctx, std::vector<EwDesc>& v);
// The Pade numerator's polynomial parts of one matrix in one pass (see blas1.cu).
struct PadeDesc {
    const double *a, *a2, *a4, *a6, *a8;
    double *b, *b6, *w, *v, *inner, *inner_even;
    size_t count;  // doubles
    int rows_p, n, cplx, degree;
    double f, f2, f4, f6;  // 2^-s and its powers (degree 13)
    double c[14];          // the Pade coefficients b_0..b_m
};
void pade_assemble_batch(Context& ctx, std::vector<PadeDesc>& v);
EwDesc ew_scaled_copy(DMat& dst, const DMat& src, double f);
EwDesc ew_add_scaled(DMat& t, const DMat& s, double f);
EwDesc ew_identity(DMat& dst, double f);
EwDesc ew_pade_split(DMat& den, DMat& num, const DMat& v, const DMat& u);
std::vector<double> norm1_batch(Context& ctx, const std::vector<const DMat*>& mats);
std::vector<double> norminf_batch(Context& ctx, const std::vector<const DMat*>& mats);
std::vector<double> abs_power_batch(Context& ctx, const std::vector<const DMat*>& mats, int p);
void panel_product_batch(Context& ctx, std::vector<PanelDesc>& v, bool cplx, bool adjoint);

// ---- elementwise and reductions (blas1.cu) ---------------------------------
void scale_inplace(Context& ctx, void* c, int m, int n, int ldc, bool cplx, double beta_re, double beta_im);
// C := beta*C on a caller's stream without a context (nothing allocated).
void scale_detached(cudaStream_t stream, double* c, int m, int n, int ldc, bool cplx, double beta_re, double beta_im);
// dst := src * f (real factor, each part scaled on its own), whole padded extent.
void scaled_copy(Context& ctx, DMat& dst, const DMat& src, double f);
// t := t + s * f
void add_scaled(Context& ctx, DMat& t, const DMat& s, double f);
// dst := f * I on the valid diagonal, zero elsewhere.
void set_identity(Context& ctx, DMat& dst, double f);
// den := v - u, num := v + u
void pade_split(Context& ctx, DMat& den, DMat& num, const DMat& v, const DMat& u);
// Norms of the valid rows x cols block, returned to the host (synchronises).
double norm1(Context& ctx, const DMat& a);
double norminf(Context& ctx, const DMat& a);
double normfro(Context& ctx, const DMat& a);
// ||abs(A)^p||_1 without forming the power (MatrixExponential.cs:468-505).
double one_norm_abs_power(Context& ctx, const DMat& a, int p);
// Y := A X or A^H X for an n x t panel of device memory (x, y with leading
// dimensions ldx, ldy in elements), in the reference's summation order.
void panel_product(Context& ctx, const DMat& a, const double* x, int ldx, double* y, int ldy, int t, bool adjoint);
// dst := src^H (transpose for real) over the padded extents.
void conj_transpose(Context& ctx, DMat& dst, const DMat& src);
// Add delta to the valid diagonal.
void shift_diagonal(Context& ctx, DMat& a, double dre, double dim);
// Sum of the valid diagonal, to the host.
void trace(Context& ctx, const DMat& a, double* re, double* im);

// ---- LU and triangular solves (lu.cu) ------------------------------------
struct LuResult {
    int singular_column = -1;
    double smallest_pivot = 0.0, largest_pivot = 0.0;
};
// In-place LU of the valid m x n block of a (padded). d_piv: device int[min(m,n)].
LuResult getrf(Context& ctx, DMat& a, int m, int n, int nb, int* d_piv);
// The reference's default block size (Lu.DefaultBlockSizeFor, Lu.cs:221-222).
int reference_block_size(int m, int n);
// A batch of independent factorizations, advanced block step by block step in
// lockstep (one launch per phase per step). d_sing receives the first
// singular column, or INT_MAX.
struct LuItem {
    DMat* a;
    int m, n, nb;
    int* d_piv;
    int* d_sing;
};
void getrf_batch(Context& ctx, std::vector<LuItem>& items);
struct SolveItem {
    const DMat* lu;
    const int* d_piv;
    DMat* b;
    int nrhs;
};
void getrs_batch(Context& ctx, std::vector<SolveItem>& items, bool adjoint);
// B := A^-1 B or A^-H B from factors (valid n x n), in place on the valid rows of b.
void getrs(Context& ctx, const DMat& lu, const int* d_piv, DMat& b, int nrhs, bool adjoint);
// The same solves in no particular order: 64-row triangular blocks and DMMA
// GEMM updates of the rows beyond them (for the precision form, whose
// refinement and condition estimate have no reference order to keep).
// d_piv null: factors without row interchanges.
void getrs_free_order(Context& ctx, const DMat& lu, const int* d_piv, DMat& b, int nrhs, bool adjoint);
// The triangular solves of the reference's kernel seam (KernelEntry.cs:98-173,
// Triangular.cs) in its order of operations: B := T^-1 B or T^-T B in place
// for the triangle of f named by kind (real); complex: the unit lower, upper
// and their adjoints (BlockedLu.cs:283-373), "transposed" meaning the
// conjugate transpose.
enum class TriangularKind { kUpper, kUpperTransposed, kLower, kLowerTransposed, kLowerUnit, kLowerUnitTransposed };
void solve_triangular(Context& ctx, TriangularKind kind, const DMat& f, DMat& b, int nrhs);

// The precision form of the solve: LU whose trailing updates (depth 512) run
// on the split-precision product with `moduli` moduli, panels of 512 columns
// factored by getrf_batch; pivots absolute. Then FP64 iterative refinement.
void getrf_mixed(Context& ctx, DMat& a, int* d_piv, int moduli);
struct MixedInfo {
    int moduli = 0, factorizations = 0, iterations = 0;
    double backward_error = 0.0, rcond = 0.0;
    int pivoting = 0;  // 1: the partial-pivoting factorization ran (the butterfly route declined)
};
// x := A^-1 b (x shaped as b). moduli 0: from the condition estimate. First
// by random butterfly transforms and elimination without pivoting; when that
// meets a zero pivot or its refinement does not reach an FP64 backward error,
// again with partial pivoting.
void gesv_mixed(Context& ctx, const DMat& a, const DMat& b, DMat& x, int moduli, int max_iter, MixedInfo& info);

// ---- algorithms (algos.cu) -------------------------------------------------
struct NormestResult {
    double value = 0.0;
    int iterations = 0, products = 0;
};
NormestResult normest_power(Context& ctx, const DMat& a, int power, int t, int itmax, int seed);
// free_order: the probes' solves by getrs_free_order (no reference order to
// keep: the precision form's condition estimate).
NormestResult normest_lu_inverse(Context& ctx, const DMat& lu, const int* d_piv, int t, int itmax, int seed,
                                 bool free_order = false);
// ||M||_1 estimate of an operator M of order n given as an in-place device
// solve: solve(panel, cols, adjoint) replaces the panel's first cols columns
// (rows >= n, zero below row n) by M x or M^H x.
NormestResult normest_solve(Context& ctx, int n, int rows, bool cplx,
                            const std::function<void(DMat&, int, bool)>& solve, int t, int itmax, int seed);

struct ExpmInfo {
    int degree = 0, squarings = 0;
};
// result := exp(a) for the valid n x n block (n >= 2).
void expm(Context& ctx, const DMat& a, DMat& result, ExpmInfo* info);
// The same for a batch of matrices of any orders >= 2, one launch per phase.
// With `on_final`, each matrix's result is handed over (moved out, its slot in
// `results` left empty) as soon as it is final -- after the Pade solve for
// s = 0, else after its last squaring -- while the others still square; the
// result is complete once the context's stream reaches the point of the call.
void expm_batch(Context& ctx, const std::vector<const DMat*>& inputs, std::vector<DMat>& results,
                std::vector<ExpmInfo>& infos, const std::function<void(size_t, DMat&&)>& on_final = {});

struct ExpmvInfo {
    int degree = 0, scaling = 0, applications = 0, early_exits = 0;
};
// exp(tA)B for dense A (MatrixExponentialAction.Dense + Run): the parameters
// on the host, the Taylor recurrence in the fused device kernel (a batch of one).
void expmv(Context& ctx, const DMat& a, const DMat& b, double t, DMat& result, ExpmvInfo* info);
// The same for a batch of independent (A_k, B_k), every B_k with the same
// column count; the Taylor recurrences of all matrices run in one cooperative
// launch (expmv_batched.cu).
// select_only_cols > 0: only (m, s) for panels of that many columns (bs is
// not read, no results).
void expmv_batch(Context& ctx, const std::vector<const DMat*>& as, const std::vector<const DMat*>& bs, double t,
                 std::vector<DMat>& results, std::vector<ExpmvInfo>& infos, int select_only_cols = 0);
// The earlier host-driven form of the dense path: every application a panel
// product launch, the norms read back to the host (kept as the reference
// point for the fused kernel, and for panels wider than it takes).
void expmv_host_loop(Context& ctx, const DMat& a, const DMat& b, double t, DMat& result, ExpmvInfo* info);
void expmv_taylor_host(Context& ctx, const DMat& shifted, const DMat& b, double t, int m, int s, double eta_re,
                       double eta_im, DMat& result, ExpmvInfo* info);
// MatrixExponentialAction.SelectParameters (:347-398).
void expmv_select_parameters(double scaled_norm, const std::function<double(int)>* alpha, double scale, int cols,
                             int& m, int& s);
// normest1 (t = 2, itmax = 5, the default seed) of A_k^p_k for a set of
// (matrix, power) items, every estimator's product step in one launch.
std::vector<double> power_norm_estimates(Context& ctx, const std::vector<const DMat*>& mats,
                                         const std::vector<int>& powers);
// The matrix-free form: y := A x by a caller's function on device panels.
using ApplyFn = int (*)(void* user, int ncols, const double* x, double* y, int ld, void* stream);
void expmv_operator(Context& ctx, int n, ApplyFn apply, void* user, const DMat& b, double t, double bound,
                    DMat& result, ExpmvInfo* info);
// normest1 of a caller's operator, through its apply and adjoint callbacks.
NormestResult normest_operator(Context& ctx, int n, bool cplx, ApplyFn apply, ApplyFn adjoint, void* user, int t,
                               int itmax, int seed);

// ---- Frechet derivative and adjoint (frechet.cu) -----------------------------
// exp(a) and, for a direction e, L(a, e) = d/dh exp(a + h e) at h = 0.
void expm_frechet(Context& ctx, const DMat& a, const DMat& e, DMat* expa, DMat& l, ExpmInfo* info);
// For F = exp(t a) b and loss = ||F - y||_F^2: the loss, F, and the gradients
// dloss/da (n x n), dloss/db (n x c) and dloss/dt (complex: the gradients of a
// real function with respect to Re and Im, as one complex matrix).
struct GradientResult {
    double loss = 0.0, grad_t = 0.0;
    ExpmInfo info;
};
GradientResult expmv_gradient(Context& ctx, const DMat& a, const DMat& b, const DMat& y, double t, DMat* f,
                              DMat& grad_a, DMat& grad_b);

}  // namespace tns
