// Split-precision products: FP64 (real or complex) C := A B (+ C) computed
// from 8-bit integer residues on the tcgen05 tensor cores, with exact 32-bit
// integer accumulation and a Chinese-remainder reconstruction in FP64
// (the modular form of the Ozaki scheme).
//
// Integers. Every row i of A is scaled by 2^(t - e_i), every column j of B by
// 2^(t - f_j), where 2^e bounds the row's (column's) largest magnitude from
// above (complex: the larger of |Re| and |Im|, shared by both parts), and
// rounded to the nearest integer: A' = rint(A 2^(t-e)), |A'| <= 2^t. Both steps
// are exact in FP64 (a power-of-two scaling, then rint), so the only error of
// the scheme is this rounding, 1/2 in the last of t bits of the row's scale.
// Residues. For each of N pairwise coprime moduli p <= 256 (256, 255, 253,
// 251, 247, 241, ... -- their prime factors are disjoint), A' mod p and
// B' mod p are taken exactly (as symmetric residues, |r| <= 128, in 8 bits).
// Products. For each modulus, R = (A' mod p)(B' mod p) is one 8-bit GEMM with
// exact 32-bit accumulation (|r|^2 K' < 2^31); R mod p = (A'B') mod p. t is
// the largest value with 2 K' 2^(2t) < P = prod(p), so A'B' is the unique
// residue class representative in (-P/2, P/2).
// Reconstruction. With u_q = (R_q y_q) mod p_q, y_q = (P/p_q)^-1 mod p_q,
// A'B' / P = frac(sum_q u_q / p_q) (the representative in [-1/2, 1/2]). All
// 1/p_q share one binary exponent, so with 1/p_q written as three aligned
// 39-bit digits the sum is three exact FP64 integer sums; the fraction of the
// leading one is exact, the trailing ones join in double-double, and
// A'B' = frac * P, then C = A'B' 2^(e_i + f_j - 2t). The reconstruction's own
// error, below 2^-110 of P, is far under the rounding of A' and B'.
// Complex. With the real and imaginary parts sharing their exponents, the
// complex product is the single real product
//     [Ar Ai] * [[Br, Bi], [-Bi, Br]]   (columns of the right factor interleaved,
// so that output columns 2j, 2j+1 are Re, Im of C[:, j]) -- four real
// multiplications per complex multiply-add, as the 4M method (never 3M).
//
// Kernels. Residues: one thread per 8 bytes of a residue row, all moduli.
// Product: one CTA per 128 x 256 output tile and all moduli: a TMA producer
// warp streams 128- and 256-row x 128-byte residue tiles (128-byte swizzle)
// through a 4-stage mbarrier ring; one thread issues tcgen05.mma kind::i8
// (M = 128, N = 256, K = 32) into one of two TMEM accumulators (all 512
// columns); four epilogue warps reduce each
// finished accumulator to u_q (tcgen05.ld) and store it as a byte plane while
// the next modulus' MMAs run. When the 256-column tiles fill the GPU, two
// CTAs of a cluster share each M = 256 MMA instead (cta_group::2): each loads
// its own 128 rows of A and half of B, so a stage is 32 KB per SM and six are
// in flight (modular_gemm_pair_kernel). Every wait is bounded; TMEM is
// released on every path. Reconstruction: one CTA per 32 x 32 output tile,
// all planes staged in shared memory, one column of 32 rows per warp store.
//
// Accuracy: each entry differs from the exact product by at most about
// K 2^-t of its row scale times its column scale (A' and B' rounded), the
// split-precision form's only error; with 20 moduli and K' <= 2048, t = 71.
// It does not reproduce the reference's rounding.

#include "batch.cuh"
#include "device_util.cuh"
#include "tcgen05.cuh"
#include "tns_internal.h"
#include "autotune.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <string>
#include <vector>

namespace tns {

namespace {

constexpr int kMaxModuli = 22;
// Pairwise coprime, largest first: 2^8, 3*5*17, 11*23, 251, 13*19, then primes
// and 7*31.
constexpr int kModuli[kMaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223,
                                     217, 211, 199, 197, 193, 191, 181, 179, 173, 167, 163};

constexpr int kTile = 128;       // output tile rows (the MMA's M); rows of an A residue tile
// Output tile columns (the MMA's N, the rows of a B residue tile): 256 when a
// launch's tiles fill the GPU (each A tile then feeds twice the columns),
// else 128.
constexpr int kKb = 128;         // bytes (8-bit elements) of K per stage
constexpr int kStages = 4;
template <int TN>
__host__ __device__ constexpr uint32_t stage_bytes() { return (uint32_t)(kTile + TN) * kKb; }  // A and B tiles
constexpr int kSplitThreads = 192;                  // producer, MMA, 4 epilogue warps
template <int TN>
constexpr int split_smem() { return kStages * (int)stage_bytes<TN>() + 1024 + 256; }

enum : int { kErrSplitFull = 11, kErrSplitEmpty = 12, kErrSplitAcc = 13, kErrSplitDrain = 14 };

// The moduli of one product form and the constants of its reconstruction.
struct CrtParams {
    int nm;                       // moduli used
    int t;                        // integer bits of the scaled operands
    int p[kMaxModuli];            // moduli
    int y[kMaxModuli];            // (P / p)^-1 mod p
    // The product epilogue's constants: with R = h 2^16 + l, u = (h w16 + l w0) mod p,
    // w0 = y mod p and w16 = 2^16 y mod p (symmetric), l w0 formed from l + 2^23
    // as fma(l + 2^23, w0, -2^23 w0).
    float w0[kMaxModuli], w16[kMaxModuli], w0_off[kMaxModuli];
    float inv[kMaxModuli];        // 1/p rounded to FP32
    // 1/p = d1 2^-47 + d2 2^-86 + d3 2^-125 (+ under 2^-125), each digit an
    // integer below 2^40: every 1/p lies in [2^-8, 2^-7), so the digits of all
    // moduli are aligned and sum_q u_q d_q stays an exact FP64 integer.
    double d1[kMaxModuli], d2[kMaxModuli], d3[kMaxModuli];
    double P_hi, P_lo;            // P = prod p as a double-double
};

// ---- exponents ---------------------------------------------------------------

// 2^e with e the least integer such that every |x| < 2^e (0 for an all-zero set).
__device__ __forceinline__ int bound_exponent(double m) { return m > 0.0 ? ilogb(m) + 1 : 0; }

struct ExpDesc {
    const double* a;  // column-major, ld elements
    int ld, rows, cols;
    int* out;
};

// Row exponents of A: one thread per (row, chunk of kRowExpChunk columns),
// the exponents of the chunks with a nonzero entry folded by atomicMax into
// out (set to INT_MIN first by exponent_init_kernel), then INT_MIN (an
// all-zero row) replaced by 0, bound_exponent's value for zero
// (exponent_fix_kernel). bound_exponent is increasing on positive values, so
// the largest chunk exponent is the exponent of the row's largest magnitude.
constexpr int kRowExpChunk = 64;

__global__ void exponent_init_kernel(const __grid_constant__ Batch<ExpDesc> b) {
    const ExpDesc& d = batch_item(b, blockIdx.y);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.rows) d.out[i] = INT_MIN;
}

__global__ void exponent_fix_kernel(const __grid_constant__ Batch<ExpDesc> b) {
    const ExpDesc& d = batch_item(b, blockIdx.y);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.rows && d.out[i] == INT_MIN) d.out[i] = 0;
}

template <bool CPLX>
__global__ void row_exponent_kernel(const __grid_constant__ Batch<ExpDesc> b) {
    const ExpDesc& d = batch_item(b, blockIdx.z);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k0 = blockIdx.y * kRowExpChunk;
    if (i >= d.rows || k0 >= d.cols) return;
    const int k1 = min(d.cols, k0 + kRowExpChunk);
    double m = 0.0;
    // Eight columns' loads in flight per step; the maximum is order-free.
    int k = k0;
    for (; k + 8 <= k1; k += 8) {
        if (CPLX) {
            double2 z[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) z[u] = reinterpret_cast<const double2*>(d.a)[(size_t)(k + u) * d.ld + i];
#pragma unroll
            for (int u = 0; u < 8; ++u) m = fmax(m, fmax(fabs(z[u].x), fabs(z[u].y)));
        } else {
            double z[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) z[u] = d.a[(size_t)(k + u) * d.ld + i];
#pragma unroll
            for (int u = 0; u < 8; ++u) m = fmax(m, fabs(z[u]));
        }
    }
    for (; k < k1; ++k) {
        if (CPLX) {
            const double2 z = reinterpret_cast<const double2*>(d.a)[(size_t)k * d.ld + i];
            m = fmax(m, fmax(fabs(z.x), fabs(z.y)));
        } else {
            m = fmax(m, fabs(d.a[(size_t)k * d.ld + i]));
        }
    }
    if (m > 0.0) atomicMax(d.out + i, bound_exponent(m));
}

// Column exponents of B: one warp per column.
template <bool CPLX>
__global__ void col_exponent_kernel(const __grid_constant__ Batch<ExpDesc> b) {
    const ExpDesc& d = batch_item(b, blockIdx.y);
    const int j = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (j >= d.cols) return;
    double m = 0.0;
    for (int k = lane; k < d.rows; k += 32) {
        if (CPLX) {
            const double2 z = reinterpret_cast<const double2*>(d.a)[(size_t)j * d.ld + k];
            m = fmax(m, fmax(fabs(z.x), fabs(z.y)));
        } else {
            m = fmax(m, fabs(d.a[(size_t)j * d.ld + k]));
        }
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) d.out[j] = bound_exponent(m);
}

// ---- residues ----------------------------------------------------------------------

// Digits. y = v 2^shift (|y| < 2^t) is written as rint(y) = sum_{i<ND} c_i 2^(14 i)
// with symmetric digits |c_i| <= 2^13, taken from the top in FP64: c_i is
// rint(x 2^-14i) (adding 1.5 2^52 rounds to an integer and leaves it in the low
// word), then x -= c_i 2^14i, which is exact (x keeps at most 53 significant
// bits: it is a multiple of y's last bit and below 2^(14i - 1)). The last digit
// rounds what is left, so the digits sum to rint(y) exactly. ND = 6 covers
// t <= 83, ND = 7 covers t <= 97.
//
// Residues. For each modulus, s = sum_i c_i w_i with w_i the symmetric residue
// of 2^(14 i) mod p (|w_i| <= 128) is an exact FP32 integer (|s| <= 2^13 +
// (ND - 1) 2^20 < 0.8 2^23), congruent to rint(y) mod p. Then r = s - p rint(s/p)
// with the quotient taken as s * fl(1/p) rounded to an integer by adding
// 1.5 2^23: the product is off s/p by under |s| 2^-24 / p < 0.4 / p, and for odd
// p the quotient s/p is at least 1/(2p) from a tie, so the rounding is the
// exact one and r lies in [-(p-1)/2, (p-1)/2] (p = 256: 1/p is exact and r in
// [-128, 128], 128 and -128 being the same byte). r + 1.5 2^23 holds r in the
// low byte of its bit pattern. Two entries go through each FP32 instruction
// (the f32x2 forms); the reduction never touches the FP64 pipe.
constexpr int kDigitBits = 14;
constexpr int kMaxDigits = 7;
constexpr double kRoundMagic = 6755399441055744.0;  // 1.5 * 2^52
constexpr float kRoundMagicF = 12582912.0f;          // 1.5 * 2^23
constexpr int kRoundMagicBits = 0x4B400000;          // bit pattern of 1.5 * 2^23

__host__ __device__ constexpr double pow2_const(int k) {
    double r = 1.0;
    for (; k > 0; --k) r *= 2.0;
    for (; k < 0; ++k) r *= 0.5;
    return r;
}

int digits_for(int t) { return t <= kDigitBits * 5 + kDigitBits - 1 ? 6 : 7; }

struct ResidueTable {
    float2 w[kMaxModuli][kMaxDigits];  // {w, w}: symmetric residue of 2^(14 i) mod p
    float2 inv[kMaxModuli];            // {1/p, 1/p} rounded to FP32
    float2 negp[kMaxModuli];           // {-p, -p}
};

constexpr ResidueTable make_residue_table() {
    ResidueTable t{};
    for (int q = 0; q < kMaxModuli; ++q) {
        const int p = kModuli[q];
        long long r = 1 % p;
        for (int i = 0; i < kMaxDigits; ++i) {
            const long long s = 2 * r > p ? r - p : r;
            t.w[q][i] = float2{(float)s, (float)s};
            for (int b = 0; b < kDigitBits; ++b) r = r * 2 % p;
        }
        const float inv = (float)(1.0 / p);
        t.inv[q] = float2{inv, inv};
        t.negp[q] = float2{(float)-p, (float)-p};
    }
    return t;
}
__constant__ ResidueTable kResidueTable = make_residue_table();

// 2^k as a double, |k| <= 1022.
__device__ __forceinline__ double pow2(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

// Digits of rint(v 2^shift) as FP32 bit patterns of 1.5 2^23 + c_i. The scale
// goes in two exact power-of-two factors (shift can exceed the exponent range
// of one double; a product that underflows belongs to an entry whose integer
// image is 0 either way).
template <int ND>
__device__ __forceinline__ void digits_of(double v, double f1, double f2, float (&c)[ND]) {
    double x = (v * f1) * f2;
#pragma unroll
    for (int i = ND - 1; i >= 1; --i) {
        const double tm = fma(x, pow2_const(-kDigitBits * i), kRoundMagic);
        c[i] = __int_as_float(__double2loint(tm) + kRoundMagicBits);
        x = fma(-(tm - kRoundMagic), pow2_const(kDigitBits * i), x);
    }
    c[0] = __int_as_float(__double2loint(x + kRoundMagic) + kRoundMagicBits);
}

__device__ __forceinline__ uint32_t pack4(uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3) {
    return __byte_perm(__byte_perm(b0, b1, 0x0040), __byte_perm(b2, b3, 0x0040), 0x5410);
}
// Byte-wise two's complement negation (no carries between bytes).
__device__ __forceinline__ uint32_t neg_bytes(uint32_t w) {
    const uint32_t n = ~w;
    return ((n & 0x7f7f7f7fu) + 0x01010101u) ^ (n & 0x80808080u);
}

// 2 NP consecutive entries of one residue row (8 or 16): their digits (in
// pairs), then for each modulus the residue bytes, handed to store(q, words)
// as NP / 2 words (uint2 or uint4).
template <int ND, int NP>
struct RowDigits {
    float2 c[ND][NP];

    template <class Load>
    __device__ __forceinline__ void take(Load load, int shift) {
        const int h = shift >> 1;
        const double f1 = pow2(h), f2 = pow2(shift - h);
        const float2 neg_magic = make_float2(-kRoundMagicF, -kRoundMagicF);
        // All the entries' loads first, so that they are in flight together.
        double v[2 * NP];
#pragma unroll
        for (int e = 0; e < 2 * NP; ++e) v[e] = load(e);
#pragma unroll
        for (int e = 0; e < NP; ++e) {
            float d0[ND], d1[ND];
            digits_of<ND>(v[2 * e], f1, f2, d0);
            digits_of<ND>(v[2 * e + 1], f1, f2, d1);
#pragma unroll
            for (int i = 0; i < ND; ++i) c[i][e] = __fadd2_rn(make_float2(d0[i], d1[i]), neg_magic);
        }
    }

    template <class Store>
    __device__ __forceinline__ void residues(int nm, Store store) const {
        const float2 magic = make_float2(kRoundMagicF, kRoundMagicF);
        const float2 neg_magic = make_float2(-kRoundMagicF, -kRoundMagicF);
        // One modulus per trip (not unrolled over the moduli: the unrolled
        // body outgrew the instruction cache); the constants are uniform
        // constant-bank loads.
#pragma unroll 1
        for (int q = 0; q < nm; ++q) {
            uint32_t b[2 * NP];
#pragma unroll
            for (int e = 0; e < NP; ++e) {
                float2 s = c[0][e];
#pragma unroll
                for (int i = 1; i < ND; ++i) s = __ffma2_rn(c[i][e], kResidueTable.w[q][i], s);
                const float2 t = __fadd2_rn(__ffma2_rn(s, kResidueTable.inv[q], magic), neg_magic);
                const float2 r = __fadd2_rn(__ffma2_rn(t, kResidueTable.negp[q], s), magic);
                b[2 * e] = __float_as_uint(r.x);
                b[2 * e + 1] = __float_as_uint(r.y);
            }
            if constexpr (NP == 8) {
                uint4 words;
                words.x = pack4(b[0], b[1], b[2], b[3]);
                words.y = pack4(b[4], b[5], b[6], b[7]);
                words.z = pack4(b[8], b[9], b[10], b[11]);
                words.w = pack4(b[12], b[13], b[14], b[15]);
                store(q, words);
            } else {
                uint2 words;
                words.x = pack4(b[0], b[1], b[2], b[3]);
                words.y = pack4(b[4], b[5], b[6], b[7]);
                store(q, words);
            }
        }
    }
};

struct ResDesc {
    const double* src;  // A (rows x k) or B (k x cols), column-major, ld elements
    int ld, m, k;       // logical rows (A) or columns (B); depth
    int kh;             // complex: offset of the imaginary half in a residue row (k rounded up to 16)
    int rows_p, kp;     // padded residue extents: rows of a plane, bytes per row
    const int* e;       // exponents of the rows (A) or columns (B)
    int8_t* dst;        // nm x rows_p x kp
};

// A' planes: row i holds [Re A(i,:), 0.., Im A(i,:), 0..] with the imaginary
// half at kh (real: A(i,:)), zeros to kp; every modulus. A thread converts 8
// entries; the four lanes of a row's 32-byte segment are adjacent, so each
// warp store writes eight whole 32-byte sectors (8 rows x 32 bytes), and the
// small per-thread state (48 digit registers) leaves room for twice the
// warps per SM of a 16-entry thread.
template <bool CPLX, int ND>
__global__ void __launch_bounds__(128) residue_a_kernel(const __grid_constant__ Batch<ResDesc> b,
                                                        const __grid_constant__ CrtParams cp) {
    const ResDesc& d = batch_item(b, blockIdx.z);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + warp * 8 + (lane >> 2);
    const int c0 = blockIdx.y * 32 + (lane & 3) * 8;
    if (i >= d.rows_p || c0 >= d.kp) return;
    const int shift = cp.t - (i < d.m ? d.e[i] : 0);
    const bool imag = CPLX && c0 >= d.kh;
    const int k0 = imag ? c0 - d.kh : c0;
    const bool rows_live = i < d.m && (!CPLX || c0 < 2 * d.kh);
    RowDigits<ND, 4> g;
    g.take(
        [&](int u) {
            const int k = k0 + u;
            if (!rows_live || k >= d.k) return 0.0;
            return CPLX ? d.src[((size_t)k * d.ld + i) * 2 + (imag ? 1 : 0)] : d.src[(size_t)k * d.ld + i];
        },
        shift);
    int8_t* row = d.dst + (size_t)i * d.kp + c0;
    const size_t plane = (size_t)d.rows_p * d.kp;
    g.residues(cp.nm, [&](int q, uint2 w) { *reinterpret_cast<uint2*>(row + q * plane) = w; });
}

// B' planes, K-major rows of the right factor. Complex: row 2j =
// [Re B(:,j); -Im B(:,j)], row 2j+1 = [Im B(:,j); Re B(:,j)] (halves at 0 and
// kh); real: row j = B(:,j); zeros to kp. One thread per 8 entries of one part
// of one column, consecutive threads on consecutive entries (whole sectors
// per warp store): a real-part thread writes them to row 2j at 0 and to row
// 2j+1 at kh, an imaginary-part thread to row 2j+1 at 0 and, negated, to row
// 2j at kh (the residues of -x are the negated residues of x). Threads past
// the last chunk write the zero tail [2 kh, kp) of both rows.
template <bool CPLX, int ND>
__global__ void __launch_bounds__(128) residue_b_kernel(const __grid_constant__ Batch<ResDesc> b,
                                                        const __grid_constant__ CrtParams cp) {
    const ResDesc& d = batch_item(b, blockIdx.y);
    constexpr int DPE = CPLX ? 2 : 1;
    const int half = (CPLX ? d.kh : d.kp) / 8;  // data chunks of one part
    const int items = CPLX ? 2 * half + (d.kp - 2 * d.kh) / 8 : half;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int jrows = d.rows_p / DPE;
    if (idx >= (long long)items * jrows) return;
    const int j = (int)(idx / items), it = (int)(idx % items);
    const bool live = j < d.m;
    int8_t* row0 = d.dst + (size_t)(DPE * j) * d.kp;
    const size_t plane = (size_t)d.rows_p * d.kp;
    if (CPLX && it >= 2 * half) {  // zero tail of both rows
        const int c0 = 2 * d.kh + (it - 2 * half) * 8;
        for (int q = 0; q < cp.nm; ++q) {
            *reinterpret_cast<uint2*>(row0 + q * plane + c0) = make_uint2(0, 0);
            *reinterpret_cast<uint2*>(row0 + q * plane + d.kp + c0) = make_uint2(0, 0);
        }
        return;
    }
    const bool imag = CPLX && it >= half;
    const int k0 = (imag ? it - half : it) * 8;
    const int shift = cp.t - (live ? d.e[j] : 0);
    RowDigits<ND, 4> g;
    g.take(
        [&](int u) {
            const int k = k0 + u;
            if (!live || k >= d.k) return 0.0;
            return CPLX ? d.src[((size_t)j * d.ld + k) * 2 + (imag ? 1 : 0)] : d.src[(size_t)j * d.ld + k];
        },
        shift);
    if (!CPLX) {
        g.residues(cp.nm, [&](int q, uint2 w) { *reinterpret_cast<uint2*>(row0 + q * plane + k0) = w; });
    } else if (!imag) {
        g.residues(cp.nm, [&](int q, uint2 w) {
            *reinterpret_cast<uint2*>(row0 + q * plane + k0) = w;
            *reinterpret_cast<uint2*>(row0 + q * plane + d.kp + d.kh + k0) = w;
        });
    } else {
        g.residues(cp.nm, [&](int q, uint2 w) {
            *reinterpret_cast<uint2*>(row0 + q * plane + d.kp + k0) = w;
            *reinterpret_cast<uint2*>(row0 + q * plane + d.kh + k0) = make_uint2(neg_bytes(w.x), neg_bytes(w.y));
        });
    }
}

// ---- the products, one per modulus ---------------------------------------------------

struct ModDesc {
    int kp;                  // bytes per residue row (multiple of 128)
    int np;                  // columns of an output plane (multiple of 128)
    int mp;                  // rows of an output plane (multiple of 128)
    int tiles_m, tile_begin;
    uint8_t* u;              // nm planes of mp x np bytes, row-major: u_q of each product entry
    int m_base;              // first output row of the tiles (a strip left over by the CTA-pair kernel)
};
struct ModMaps {
    CUtensorMap a, b;  // residues as (kp bytes) x (rows) x nm; boxes of 128 bytes x 128 (A) or 256 (B) rows, 128-byte swizzle
};

// One CTA's work on output tile `tile` of the launch's tile list.
template <int TN>
__device__ __forceinline__ void modular_tile(const ModDesc* __restrict__ descs, const ModMaps* __restrict__ maps,
                                             int nprob, const CrtParams& cp, int* err, int tile) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    constexpr uint32_t kStageBytes = stage_bytes<TN>();
    constexpr uint32_t kTmemCols = 2 * TN;  // two accumulators (power of two >= 32)
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
    uint64_t* empty = full + kStages;
    uint64_t* accf = empty + kStages;   // accumulator b is complete (MMA -> epilogue)
    uint64_t* acce = accf + 2;          // accumulator b is free again (epilogue -> MMA)
    uint64_t* done = acce + 2;          // every MMA issued has completed (for the exit)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    uint32_t* consumed = tmem_slot + 1;  // stages the MMA thread consumed

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (descs[mid].tile_begin <= tile) lo = mid;
        else hi = mid - 1;
    }
    const ModDesc& D = descs[lo];
    const ModMaps& MP = maps[lo];
    const int local = tile - D.tile_begin;
    const int m0 = D.m_base + (local % D.tiles_m) * kTile, n0 = (local / D.tiles_m) * TN;
    const int nkb = D.kp / kKb;
    const int nm = cp.nm;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], 4);
        }
        mbar_init(done, 1);
        *consumed = 0;
        mbar_fence_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    auto stage_a = [&](int s) { return smem + s * kStageBytes; };
    auto stage_b = [&](int s) { return smem + s * kStageBytes + kTile * kKb; };

    uint32_t issued = 0;  // producer's stage count
    if (warp == 0) {
        if (lane == 0) {
            tensormap_acquire(&MP.a);
            tensormap_acquire(&MP.b);
            bool ok = true;
            for (int q = 0; q < nm && ok; ++q) {
                for (int kb = 0; kb < nkb; ++kb) {
                    const int st = issued % kStages;
                    if (!mbar_wait_bounded(&empty[st], ((issued / kStages) & 1) ^ 1, err, kErrSplitEmpty)) {
                        ok = false;
                        break;
                    }
                    mbar_arrive_expect_tx(&full[st], kStageBytes);
                    tma_load_3d(stage_a(st), &MP.a, kb * kKb, m0, q, &full[st]);
                    tma_load_3d(stage_b(st), &MP.b, kb * kKb, n0, q, &full[st]);
                    ++issued;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = i8_instr_desc(kTile, TN);
            uint32_t it = 0;
            bool ok = true;
            for (int q = 0; q < nm && ok; ++q) {
                const int buf = q & 1;
                if (!mbar_wait_bounded(&acce[buf], ((q >> 1) & 1) ^ 1, err, kErrSplitAcc)) break;
                tc_fence_after_sync();
                const uint32_t dacc = tmem + buf * TN;
                for (int kb = 0; kb < nkb; ++kb) {
                    const int st = it % kStages;
                    if (!mbar_wait_bounded(&full[st], (it / kStages) & 1, err, kErrSplitFull)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after_sync();
#pragma unroll
                    for (int kk = 0; kk < kKb / 32; ++kk) {
                        mma_i8(dacc, sw128_kmajor_desc(stage_a(st), kk * 32), sw128_kmajor_desc(stage_b(st), kk * 32),
                               idesc, !(kb == 0 && kk == 0));
                    }
                    mma_commit(&empty[st]);
                    ++it;
                }
                if (ok) mma_commit(&accf[buf]);
            }
            *consumed = it;
            mma_commit(done);
        }
    } else {
        // Epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (the rows of the
        // tile) and stores u_q = (R mod p) y mod p as one byte per entry.
        const int quarter = warp & 3;
        const int row = quarter * 32 + lane;
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        for (int q = 0; q < nm; ++q) {
            const int buf = q & 1;
            // The TMEM moves below are warp-collective: the warp goes on only
            // if every lane saw the accumulator complete.
            const bool got = mbar_wait_bounded(&accf[buf], (q >> 1) & 1, err, kErrSplitAcc);
            if (!__all_sync(0xffffffffu, got)) break;
            tc_fence_after_sync();
            // u = (R y) mod p in [0, p] (p meaning 0), in FP32, two entries per
            // instruction. R = h 2^16 + l with h = R >> 16 (arithmetic) and
            // l = R & 0xffff, both read into floats through their bit patterns
            // (2^23 + l; 1.5 2^23 + h, less 1.5 2^23). s = h w16 + l w0 is an
            // exact FP32 integer, |s| <= 2^15 128 + 2^16 128 = 1.5 2^23. The
            // quotient floor(s/p) is s * fl(1/p) rounded down by adding 1.5 2^23
            // in round-toward-minus-infinity: the product is off s/p by under
            // 0.75/p, so it is the exact floor, or one less when p divides s
            // (u = p then). u + 1.5 2^23 holds u in its low byte.
            const float2 w0 = make_float2(cp.w0[q], cp.w0[q]), w16 = make_float2(cp.w16[q], cp.w16[q]);
            const float2 w0_off = make_float2(cp.w0_off[q], cp.w0_off[q]);
            const float2 inv = make_float2(cp.inv[q], cp.inv[q]);
            const float2 negp = make_float2((float)-cp.p[q], (float)-cp.p[q]);
            const float2 magic = make_float2(kRoundMagicF, kRoundMagicF);
            const float2 neg_magic = make_float2(-kRoundMagicF, -kRoundMagicF);
            uint8_t* plane = D.u + ((size_t)q * D.mp + m0 + row) * D.np + n0;
            for (int c0 = 0; c0 < TN; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + lane_addr + buf * TN + c0, v);
                tmem_wait_ld();
                uint32_t bytes[16];
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const uint32_t x0 = v[2 * e], x1 = v[2 * e + 1];
                    const float2 lm = make_float2(__uint_as_float((x0 & 0xffffu) | 0x4B000000u),
                                                  __uint_as_float((x1 & 0xffffu) | 0x4B000000u));
                    const float2 hm = make_float2(__int_as_float(((int)x0 >> 16) + kRoundMagicBits),
                                                  __int_as_float(((int)x1 >> 16) + kRoundMagicBits));
                    const float2 sv = __ffma2_rn(__fadd2_rn(hm, neg_magic), w16, __ffma2_rn(lm, w0, w0_off));
                    const float2 t = __fadd2_rn(__ffma2_rd(sv, inv, magic), neg_magic);
                    const float2 u = __fadd2_rn(__ffma2_rn(t, negp, sv), magic);
                    bytes[2 * e] = __float_as_uint(u.x);
                    bytes[2 * e + 1] = __float_as_uint(u.y);
                }
                uint4 words;
                words.x = pack4(bytes[0], bytes[1], bytes[2], bytes[3]);
                words.y = pack4(bytes[4], bytes[5], bytes[6], bytes[7]);
                words.z = pack4(bytes[8], bytes[9], bytes[10], bytes[11]);
                words.w = pack4(bytes[12], bytes[13], bytes[14], bytes[15]);
                *reinterpret_cast<uint4*>(plane + c0) = words;
            }
            tc_fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[buf]);
        }
    }

    // Leave only when nothing is in flight: every MMA done (TMEM) and every
    // stage the producer issued landed (shared memory).
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0 && lane == 0) {
        for (uint32_t j = *consumed; j < issued; ++j)
            if (!mbar_wait_bounded(&full[j % kStages], (j / kStages) & 1, err, kErrSplitDrain)) break;
    }
    if (warp == 1) {
        if (lane == 0) mbar_wait_bounded(done, 0, err, kErrSplitDrain);
        __syncwarp();
        tc_fence_after_sync();
        tmem_dealloc(tmem, kTmemCols);
    }
}

template <int TN>
__global__ void __launch_bounds__(kSplitThreads, 1)
    modular_gemm_kernel(const ModDesc* __restrict__ descs, const ModMaps* __restrict__ maps, int nprob,
                        const __grid_constant__ CrtParams cp, int* err) {
    modular_tile<TN>(descs, maps, nprob, cp, err, (int)blockIdx.x);
}

// The same product by CTA pairs (a cluster of two CTAs, cta_group::2): a pair
// owns a 256 x 256 output tile. Each CTA loads 128 rows of A and its half
// (128 rows) of B into its own shared memory, both reporting the bytes to the
// even CTA's barrier; one thread of the even CTA issues the M = 256 MMAs,
// which write 128 accumulator rows into each CTA's TMEM, and its commits
// arrive on both CTAs' barriers. Per SM a stage is 32 KB instead of 48, so six
// stages are in flight. Each CTA's epilogue reduces its own accumulator rows
// and frees the buffer on the even CTA's barrier (8 warps). Every wait is
// bounded; both CTAs meet at a cluster barrier before TMEM is released.
constexpr int kStagesPair = 6;
constexpr int kPairN = 256;                                    // output tile columns of a pair
constexpr uint32_t kPairStageBytes = (uint32_t)(kTile + kPairN / 2) * kKb;  // A rows and half of B's
constexpr int kPairSmem = kStagesPair * (int)kPairStageBytes + 1024 + 256;
constexpr uint32_t kPairTmemCols = 2 * kPairN;

static_assert(kPairSmem >= split_smem<kPairN>(), "the pair kernel's shared memory holds a one-CTA tile");

// The first CTAs (odd_tiles rounded up to a whole cluster) take the one-CTA
// tiles of odd last strips (odescs), one each, as modular_gemm_kernel<256>,
// so that they run among the first pairs instead of after the last; the
// clusters after them take the pair tiles (npairs of them).
__global__ void __launch_bounds__(kSplitThreads, 1)
    modular_gemm_pair_kernel(const ModDesc* __restrict__ descs, const ModMaps* __restrict__ maps, int nprob,
                             int npairs, const ModDesc* __restrict__ odescs, const ModMaps* __restrict__ omaps,
                             int nodd, int odd_tiles, const __grid_constant__ CrtParams cp, int* err) {
    const int solo_ctas = odd_tiles + (odd_tiles & 1);
    if ((int)blockIdx.x < solo_ctas) {  // the same for both CTAs of a cluster
        if ((int)blockIdx.x < odd_tiles) modular_tile<kPairN>(odescs, omaps, nodd, cp, err, (int)blockIdx.x);
        return;
    }
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStagesPair * kPairStageBytes);  // even CTA's are used
    uint64_t* empty = full + kStagesPair;
    uint64_t* accf = empty + kStagesPair;
    uint64_t* acce = accf + 2;  // even CTA's are used: 4 epilogue warps of each CTA arrive
    uint64_t* done = acce + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    uint32_t* consumed = tmem_slot + 1;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const int pair = ((int)blockIdx.x - solo_ctas) >> 1;
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (descs[mid].tile_begin <= pair) lo = mid;
        else hi = mid - 1;
    }
    const ModDesc& D = descs[lo];
    const ModMaps& MP = maps[lo];
    const int local = pair - D.tile_begin;
    const int m0 = (2 * (local % D.tiles_m) + (int)rank) * kTile, n0 = (local / D.tiles_m) * kPairN;
    const int nb0 = n0 + (int)rank * (kPairN / 2);  // this CTA's B rows
    const int nkb = D.kp / kKb;
    const int nm = cp.nm;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStagesPair; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], 8);
        }
        mbar_init(done, 1);
        *consumed = 0;
        mbar_fence_init();
    }
    if (warp == 1) {
        tmem_alloc2(tmem_slot, kPairTmemCols);
        tmem_relinquish2();
    }
    tc_fence_before_sync();
    __syncthreads();
    cluster_sync();  // both CTAs' barriers exist before either reaches the other's
    tc_fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    auto stage_a = [&](int s) { return smem + s * kPairStageBytes; };
    auto stage_b = [&](int s) { return smem + s * kPairStageBytes + kTile * kKb; };

    uint32_t issued = 0;
    if (warp == 0) {
        if (lane == 0) {
            tensormap_acquire(&MP.a);
            tensormap_acquire(&MP.b);
            bool ok = true;
            for (int q = 0; q < nm && ok; ++q) {
                for (int kb = 0; kb < nkb; ++kb) {
                    const int st = issued % kStagesPair;
                    if (!mbar_wait_bounded(&empty[st], ((issued / kStagesPair) & 1) ^ 1, err, kErrSplitEmpty)) {
                        ok = false;
                        break;
                    }
                    if (rank == 0) mbar_arrive_expect_tx(&full[st], 2 * kPairStageBytes);
                    const uint32_t bar = cluster_addr(&full[st], 0);
                    tma_load_3d_pair(stage_a(st), &MP.a, kb * kKb, m0, q, bar);
                    tma_load_3d_pair(stage_b(st), &MP.b, kb * kKb, nb0, q, bar);
                    ++issued;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {
            constexpr uint32_t idesc = i8_instr_desc(2 * kTile, kPairN);
            uint32_t it = 0;
            bool ok = true;
            for (int q = 0; q < nm && ok; ++q) {
                const int buf = q & 1;
                if (!mbar_wait_bounded(&acce[buf], ((q >> 1) & 1) ^ 1, err, kErrSplitAcc)) break;
                tc_fence_after_sync();
                const uint32_t dacc = tmem + buf * kPairN;
                for (int kb = 0; kb < nkb; ++kb) {
                    const int st = it % kStagesPair;
                    if (!mbar_wait_bounded(&full[st], (it / kStagesPair) & 1, err, kErrSplitFull)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after_sync();
#pragma unroll
                    for (int kk = 0; kk < kKb / 32; ++kk) {
                        mma_i8_pair(dacc, sw128_kmajor_desc(stage_a(st), kk * 32),
                                    sw128_kmajor_desc(stage_b(st), kk * 32), idesc, !(kb == 0 && kk == 0));
                    }
                    mma_commit_pair(&empty[st], 0x3);
                    ++it;
                }
                if (ok) mma_commit_pair(&accf[buf], 0x3);
            }
            *consumed = it;
            mma_commit_pair(done, 0x3);
        }
    } else {
        // Epilogue: as in modular_gemm_kernel, over this CTA's 128 accumulator
        // rows and the pair's 256 columns.
        const int quarter = warp & 3;
        const int row = quarter * 32 + lane;
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        const uint32_t acce_even[2] = {cluster_addr(&acce[0], 0), cluster_addr(&acce[1], 0)};
        for (int q = 0; q < nm; ++q) {
            const int buf = q & 1;
            const bool got = mbar_wait_bounded(&accf[buf], (q >> 1) & 1, err, kErrSplitAcc);
            if (!__all_sync(0xffffffffu, got)) break;
            tc_fence_after_sync();
            const float2 w0 = make_float2(cp.w0[q], cp.w0[q]), w16 = make_float2(cp.w16[q], cp.w16[q]);
            const float2 w0_off = make_float2(cp.w0_off[q], cp.w0_off[q]);
            const float2 inv = make_float2(cp.inv[q], cp.inv[q]);
            const float2 negp = make_float2((float)-cp.p[q], (float)-cp.p[q]);
            const float2 magic = make_float2(kRoundMagicF, kRoundMagicF);
            const float2 neg_magic = make_float2(-kRoundMagicF, -kRoundMagicF);
            uint8_t* plane = D.u + ((size_t)q * D.mp + m0 + row) * D.np + n0;
            for (int c0 = 0; c0 < kPairN; c0 += 16) {
                uint32_t v[16];
                tmem_ld16(tmem + lane_addr + buf * kPairN + c0, v);
                tmem_wait_ld();
                uint32_t bytes[16];
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const uint32_t x0 = v[2 * e], x1 = v[2 * e + 1];
                    const float2 lm = make_float2(__uint_as_float((x0 & 0xffffu) | 0x4B000000u),
                                                  __uint_as_float((x1 & 0xffffu) | 0x4B000000u));
                    const float2 hm = make_float2(__int_as_float(((int)x0 >> 16) + kRoundMagicBits),
                                                  __int_as_float(((int)x1 >> 16) + kRoundMagicBits));
                    const float2 sv = __ffma2_rn(__fadd2_rn(hm, neg_magic), w16, __ffma2_rn(lm, w0, w0_off));
                    const float2 t = __fadd2_rn(__ffma2_rd(sv, inv, magic), neg_magic);
                    const float2 u = __fadd2_rn(__ffma2_rn(t, negp, sv), magic);
                    bytes[2 * e] = __float_as_uint(u.x);
                    bytes[2 * e + 1] = __float_as_uint(u.y);
                }
                uint4 words;
                words.x = pack4(bytes[0], bytes[1], bytes[2], bytes[3]);
                words.y = pack4(bytes[4], bytes[5], bytes[6], bytes[7]);
                words.z = pack4(bytes[8], bytes[9], bytes[10], bytes[11]);
                words.w = pack4(bytes[12], bytes[13], bytes[14], bytes[15]);
                *reinterpret_cast<uint4*>(plane + c0) = words;
            }
            tc_fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(acce_even[buf]);
        }
    }

    // Leave only when nothing is in flight. The even CTA waits for the stages
    // it issued but did not consume (all bytes of both CTAs report there);
    // each CTA waits for the pair's last commit; then both meet, so neither
    // leaves while the other's MMAs or arrivals may still reach it.
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0 && lane == 0 && rank == 0) {
        for (uint32_t j = *consumed; j < issued; ++j)
            if (!mbar_wait_bounded(&full[j % kStagesPair], (j / kStagesPair) & 1, err, kErrSplitDrain)) break;
    }
    if (warp == 1 && lane == 0) mbar_wait_bounded(done, 0, err, kErrSplitDrain);
    tc_fence_before_sync();
    __syncthreads();
    cluster_sync();
    if (warp == 1) {
        tc_fence_after_sync();
        tmem_dealloc2(tmem, kPairTmemCols);
    }
}

// ---- reconstruction ----------------------------------------------------------------------

struct CrtDesc {
    const uint8_t* u;   // nm planes, mp x np row-major
    int mp, np;
    int m, n;           // output rows and (complex or real) columns
    const int* ea;      // row exponents of A
    const int* eb;      // column exponents of B
    double* c;          // column-major output (complex interleaved), ld elements
    int ldc;
    int accumulate;     // 0: C = AB, 1: C += AB
};

// A'B' / P = frac(sum_q u_q / p_q), then A'B' = frac * P. The sum is three
// exact FP64 integer sums over the aligned digits of 1/p_q; the fraction is
// taken of the leading one (exactly) and the two trailing ones are added in
// double-double.
__device__ __forceinline__ double from_digit_sums(double s1, double s2, double s3, const CrtParams& cp) {
    const double f1 = scalbn(s1 - scalbn(rint(scalbn(s1, -47)), 47), -47);  // in [-1/2, 1/2]
    const double f2 = scalbn(s2, -86), f3 = scalbn(s3, -125);
    const double fh = f1 + f2;
    const double bb = fh - f1;
    const double fl = (f1 - (fh - bb)) + (f2 - bb) + f3;
    const double r = fh * cp.P_hi;
    return r + (fma(fh, cp.P_hi, -r) + fh * cp.P_lo + fl * cp.P_hi);
}

// One CTA per 32 x 32 output tile: the tile's residue bytes of every modulus
// staged in shared memory (16-byte loads of plane rows; rows padded to an odd
// number of words so that the 32 lanes, one row each, read distinct banks),
// then warp w computes output columns w, w + 8, ..., one row per lane
// (column-major stores of 32 consecutive rows). A complex entry's Re and Im
// bytes are adjacent and read together.
template <bool CPLX>
__global__ void __launch_bounds__(256) crt_kernel(const __grid_constant__ Batch<CrtDesc> b,
                                                  const __grid_constant__ CrtParams cp) {
    const CrtDesc& d = batch_item(b, blockIdx.z);
    constexpr int DPE = CPLX ? 2 : 1;
    constexpr int TW = 32 * DPE;   // plane bytes per tile row
    constexpr int PITCH = TW + 4;  // odd number of 4-byte words
    __shared__ __align__(16) uint8_t su[kMaxModuli][32][PITCH];
    const int r0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
    if (r0 >= d.m || j0 >= d.n) return;
    const int nm = cp.nm;
    // Whole 16-byte pieces are in bounds: mp is a multiple of 128 and
    // np >= DPE * round_up(n, 32).
    constexpr int V = TW / 16;
    for (int e = threadIdx.x; e < nm * 32 * V; e += blockDim.x) {
        const int q = e / (32 * V), rr = (e / V) % 32, cv = e % V;
        const int4 w = *reinterpret_cast<const int4*>(d.u + ((size_t)q * d.mp + r0 + rr) * d.np + j0 * DPE + cv * 16);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&su[q][rr][cv * 16]);
        dst[0] = (uint32_t)w.x;
        dst[1] = (uint32_t)w.y;
        dst[2] = (uint32_t)w.z;
        dst[3] = (uint32_t)w.w;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = r0 + lane;
    if (i >= d.m) return;
    const int ei = d.ea[i];
    // The four columns' exponents and (when accumulating) old C entries are
    // loaded before the digit sums, so their latency overlaps the arithmetic.
    int sc4[4];
    double2 old4[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int j = j0 + warp + 8 * u;
        sc4[u] = j < d.n ? ei + d.eb[j] - 2 * cp.t : 0;
        old4[u] = make_double2(0.0, 0.0);
        if (d.accumulate && j < d.n) {
            if (CPLX) old4[u] = reinterpret_cast<const double2*>(d.c)[(size_t)j * d.ldc + i];
            else old4[u].x = d.c[(size_t)j * d.ldc + i];
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int jj = warp + 8 * u;
        const int j = j0 + jj;
        if (j >= d.n) break;
        const int sc = sc4[u];
        double a1 = 0.0, a2 = 0.0, a3 = 0.0, b1 = 0.0, b2 = 0.0, b3 = 0.0;
        for (int q = 0; q < nm; ++q) {
            // Bytes to doubles exactly without a conversion instruction: the
            // byte as the low word of 2^52 + byte, minus 2^52.
            double ur, ui = 0.0;
            if (CPLX) {
                const uint32_t v = *reinterpret_cast<const uint16_t*>(&su[q][lane][2 * jj]);
                ur = __hiloint2double(0x43300000, (int)(v & 0xFF)) - 4503599627370496.0;
                ui = __hiloint2double(0x43300000, (int)(v >> 8)) - 4503599627370496.0;
            } else {
                ur = __hiloint2double(0x43300000, (int)su[q][lane][jj]) - 4503599627370496.0;
            }
            a1 = fma(ur, cp.d1[q], a1);
            a2 = fma(ur, cp.d2[q], a2);
            a3 = fma(ur, cp.d3[q], a3);
            if (CPLX) {
                b1 = fma(ui, cp.d1[q], b1);
                b2 = fma(ui, cp.d2[q], b2);
                b3 = fma(ui, cp.d3[q], b3);
            }
        }
        const double re = scalbn(from_digit_sums(a1, a2, a3, cp), sc);
        if (CPLX) {
            const double im = scalbn(from_digit_sums(b1, b2, b3, cp), sc);
            double2* p = reinterpret_cast<double2*>(d.c) + (size_t)j * d.ldc + i;
            double2 r = make_double2(re, im);
            if (d.accumulate) r = make_double2(old4[u].x + r.x, old4[u].y + r.y);
            *p = r;
        } else {
            double* p = d.c + (size_t)j * d.ldc + i;
            *p = d.accumulate ? old4[u].x + re : re;
        }
    }
}

// ---- host ------------------------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }();
    if (!fn) fail(TNS_E_DEVICE, "the CUDA driver does not provide cuTensorMapEncodeTiled");
    return fn;
}

// The residues of one operand as a 3-D byte array (kp x rows_p x nm), boxes of
// 128 bytes x box_rows x 1 with 128-byte swizzle.
void encode_residues(CUtensorMap* map, const int8_t* base, int kp, int rows_p, int nm, int box_rows) {
    cuuint64_t dims[3] = {(cuuint64_t)kp, (cuuint64_t)rows_p, (cuuint64_t)nm};
    cuuint64_t strides[2] = {(cuuint64_t)kp, (cuuint64_t)kp * rows_p};
    cuuint32_t box[3] = {(cuuint32_t)kKb, (cuuint32_t)box_rows, 1};
    cuuint32_t elem[3] = {1, 1, 1};
    CUresult r = tensor_map_encoder()(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t*>(base), dims, strides,
                                      box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        fail(TNS_E_DEVICE, "TMA descriptor encoding for the split product failed (CUresult " + std::to_string((int)r) + ")");
}

int inverse_mod(int a, int p) {  // a^-1 mod p, a and p coprime
    int t = 0, nt = 1, r = p, nr = a % p;
    while (nr != 0) {
        const int qq = r / nr;
        int tmp = t - qq * nt;
        t = nt;
        nt = tmp;
        tmp = r - qq * nr;
        r = nr;
        nr = tmp;
    }
    return t < 0 ? t + p : t;
}

// Moduli and reconstruction constants for nm moduli and products of depth
// kmax (the deepest K' of the batch).
CrtParams crt_params(int nm, int kmax) {
    CrtParams cp{};
    cp.nm = nm;
    double ph = 1.0, pl = 0.0;  // P as a double-double
    for (int q = 0; q < nm; ++q) {
        const int p = kModuli[q];
        cp.p[q] = p;
        int mq = 1;  // (P / p) mod p
        for (int r = 0; r < nm; ++r)
            if (r != q) mq = (int)((long long)mq * (kModuli[r] % p) % p);
        cp.y[q] = inverse_mod(mq, p);
        auto sym = [p](long long r) { return (float)(2 * r > p ? r - p : r); };
        cp.w0[q] = sym(cp.y[q] % p);
        cp.w16[q] = sym((long long)cp.y[q] * (65536 % p) % p);
        cp.w0_off[q] = -8388608.0f * cp.w0[q];
        cp.inv[q] = (float)(1.0 / p);
        const unsigned long long d1 = (1ULL << 47) / p, r1 = (1ULL << 47) - d1 * p;
        const unsigned long long d2 = (r1 << 39) / p, r2 = (r1 << 39) - d2 * p;
        const unsigned long long d3 = (r2 << 39) / p;
        cp.d1[q] = (double)d1;
        cp.d2[q] = (double)d2;
        cp.d3[q] = (double)d3;
        const double h = ph * p;
        const double l = std::fma(ph, (double)p, -h) + pl * p;
        ph = h + l;
        pl = l - (ph - h);
    }
    cp.P_hi = ph;
    cp.P_lo = pl;
    // 2 K' 2^(2t) < P: with P >= 2^L and K' <= 2^c, 1 + c + 2t < L.
    int L = 0;
    std::frexp(ph, &L);
    L -= 1;
    int c = 0;
    while ((1LL << c) < (long long)std::max(1, kmax)) ++c;
    cp.t = std::min(96, (L - 2 - c) / 2);
    if (cp.t < 8) fail(TNS_E_ARGUMENT, "too few moduli for a split-precision product of this depth");
    return cp;
}

template <bool CPLX>
void split_launch(Context& ctx, std::vector<SplitProduct>& v, int nm) {
    constexpr int DPE = CPLX ? 2 : 1;
    struct Sizes {
        int m, n, k, kh, mp, np, kp;
        size_t a_off, b_off, u_off, ea_off, eb_off;
    };
    std::vector<Sizes> z;
    size_t total = 0;
    auto take = [&](size_t bytes) {
        size_t off = total;
        total += (bytes + 255) & ~size_t(255);
        return off;
    };
    // 256-column tiles when they fill the GPU, or as the autotuner found; a
    // trial lays out for 256 and runs both widths over the same residues.
    long long tiles_wide = 0, depth = 0;
    for (auto& p : v) {
        tiles_wide += (long long)((p.a->rows + kTile - 1) / kTile) * ((DPE * p.b->cols + 255) / 256);
        depth = std::max<long long>(depth, round_up(CPLX ? 2 * round_up(p.a->cols, 16) : p.a->cols, kKb));
    }
    const TuneKind tune_kind = CPLX ? TuneKind::kSplitComplex : TuneKind::kSplitReal;
    const int known = ctx.autotune ? tuned_variant(ctx.device, tune_kind, tiles_wide, depth) : -1;
    const bool trial = ctx.autotune && known < 0;
    const int tn = trial ? 256 : known >= 0 ? (known ? 256 : 128) : (tiles_wide >= ctx.num_sms ? 256 : 128);
    int kmax = 1;
    for (auto& p : v) {
        Sizes s{};
        s.m = p.a->rows;
        s.k = p.a->cols;
        s.n = p.b->cols;
        s.mp = round_up(s.m, kTile);
        s.np = round_up(DPE * s.n, tn);
        // complex rows: the real half, zeros to kh, the imaginary half at kh
        s.kh = CPLX ? round_up(s.k, 16) : s.k;
        s.kp = round_up(CPLX ? 2 * s.kh : s.k, kKb);
        // Exact 32-bit sums of residue products (|r| <= 128).
        if ((double)s.kp * 128.0 * 128.0 >= 2147483647.0)
            fail(TNS_E_ARGUMENT, "split-precision product too deep for exact 32-bit accumulation");
        kmax = std::max(kmax, DPE * s.k);
        s.a_off = take((size_t)nm * s.mp * s.kp);
        s.b_off = take((size_t)nm * s.np * s.kp);
        s.u_off = take((size_t)nm * s.mp * s.np);
        s.ea_off = take(sizeof(int) * s.mp);
        s.eb_off = take(sizeof(int) * std::max(1, s.n));
        z.push_back(s);
    }
    const CrtParams cp = crt_params(nm, kmax);
    char* scratch = static_cast<char*>(ctx.scratch(total));
    auto at = [&](size_t off) { return scratch + off; };

    std::vector<ExpDesc> rows, cols;
    std::vector<ResDesc> ra, rb;
    std::vector<ModDesc> md;
    std::vector<CrtDesc> cd;
    std::vector<ModMaps> maps(v.size());
    std::vector<ModDesc> md_narrow;              // a trial's 128-column tiles over the same layout
    std::vector<ModMaps> maps_narrow(trial ? v.size() : 0);
    int max_m = 0, max_cols = 0, max_rows_a = 0, max_chunks = 0, max_out_rows = 0, max_out_cols = 0;
    long long max_b_threads = 0;
    int tiles = 0, tiles_narrow = 0;
    for (size_t q = 0; q < v.size(); ++q) {
        const auto& p = v[q];
        const auto& s = z[q];
        int* ea = reinterpret_cast<int*>(at(s.ea_off));
        int* eb = reinterpret_cast<int*>(at(s.eb_off));
        int8_t* a8 = reinterpret_cast<int8_t*>(at(s.a_off));
        int8_t* b8 = reinterpret_cast<int8_t*>(at(s.b_off));
        uint8_t* u8 = reinterpret_cast<uint8_t*>(at(s.u_off));
        rows.push_back(ExpDesc{p.a->p, p.a->ld(), s.m, s.k, ea});
        cols.push_back(ExpDesc{p.b->p, p.b->ld(), s.k, s.n, eb});
        ra.push_back(ResDesc{p.a->p, p.a->ld(), s.m, s.k, s.kh, s.mp, s.kp, ea, a8});
        rb.push_back(ResDesc{p.b->p, p.b->ld(), s.n, s.k, s.kh, s.np, s.kp, eb, b8});
        md.push_back(ModDesc{s.kp, s.np, s.mp, s.mp / kTile, tiles, u8, 0});
        cd.push_back(CrtDesc{u8, s.mp, s.np, s.m, s.n, ea, eb, p.c->p, p.c->ld(), p.beta != 0.0 ? 1 : 0});
        tiles += (s.mp / kTile) * (s.np / tn);
        encode_residues(&maps[q].a, a8, s.kp, s.mp, nm, kTile);
        encode_residues(&maps[q].b, b8, s.kp, s.np, nm, tn);
        if (trial) {
            md_narrow.push_back(ModDesc{s.kp, s.np, s.mp, s.mp / kTile, tiles_narrow, u8, 0});
            tiles_narrow += (s.mp / kTile) * (s.np / 128);
            maps_narrow[q].a = maps[q].a;
            encode_residues(&maps_narrow[q].b, b8, s.kp, s.np, nm, 128);
        }
        max_m = std::max(max_m, s.m);
        max_cols = std::max(max_cols, s.n);
        max_rows_a = std::max(max_rows_a, s.mp);
        max_chunks = std::max(max_chunks, s.kp / 32);
        // residue_b: one thread per 8 entries of one part of a column of B
        // plus the zero-tail chunks
        const long long bchunks = CPLX ? 2 * (s.kh / 8) + (s.kp - 2 * s.kh) / 8 : s.kp / 8;
        max_b_threads = std::max(max_b_threads, bchunks * (s.np / DPE));
        max_out_rows = std::max(max_out_rows, s.m);
        max_out_cols = std::max(max_out_cols, s.n);
    }
    if (tiles == 0) return;
    {
        Batch<ExpDesc> br = make_batch(ctx, rows);
        exponent_init_kernel<<<dim3((max_m + 255) / 256, br.count), 256, 0, ctx.stream>>>(br);
        TNS_CUDA(cudaGetLastError());
        int max_k = 1;
        for (auto& r : rows) max_k = std::max(max_k, r.cols);
        row_exponent_kernel<CPLX><<<dim3((max_m + 127) / 128, (max_k + kRowExpChunk - 1) / kRowExpChunk, br.count),
                                    128, 0, ctx.stream>>>(br);
        TNS_CUDA(cudaGetLastError());
        exponent_fix_kernel<<<dim3((max_m + 255) / 256, br.count), 256, 0, ctx.stream>>>(br);
        ctx.kernel_launches += 2;
        TNS_CUDA(cudaGetLastError());
        Batch<ExpDesc> bc = make_batch(ctx, cols);
        col_exponent_kernel<CPLX><<<dim3((max_cols + 7) / 8, bc.count), 256, 0, ctx.stream>>>(bc);
        TNS_CUDA(cudaGetLastError());
        Batch<ResDesc> bra = make_batch(ctx, ra);
        const dim3 grid_a((max_rows_a + 31) / 32, max_chunks, bra.count);
        if (digits_for(cp.t) == 6) residue_a_kernel<CPLX, 6><<<grid_a, 128, 0, ctx.stream>>>(bra, cp);
        else residue_a_kernel<CPLX, 7><<<grid_a, 128, 0, ctx.stream>>>(bra, cp);
        TNS_CUDA(cudaGetLastError());
        Batch<ResDesc> brb = make_batch(ctx, rb);
        const dim3 grid_b((unsigned)((max_b_threads + 127) / 128), brb.count);
        if (digits_for(cp.t) == 6) residue_b_kernel<CPLX, 6><<<grid_b, 128, 0, ctx.stream>>>(brb, cp);
        else residue_b_kernel<CPLX, 7><<<grid_b, 128, 0, ctx.stream>>>(brb, cp);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches += 4;
    }
    const ModDesc* d_desc = static_cast<const ModDesc*>(ctx.upload(md.data(), sizeof(ModDesc) * md.size()));
    const ModMaps* d_maps = static_cast<const ModMaps*>(ctx.upload(maps.data(), sizeof(ModMaps) * maps.size()));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ctx.timing) {
        e0 = ctx.take_event();
        e1 = ctx.take_event();
        TNS_CUDA(cudaEventRecord(e0, ctx.stream));
    }
    auto launch = [&](auto kernel, int smem_bytes, bool& configured, const ModDesc* descs, const ModMaps* mps,
                      int ntiles, int nprob = -1) {
        if (!configured) {
            TNS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes));
            configured = true;
        }
        kernel<<<ntiles, kSplitThreads, smem_bytes, ctx.stream>>>(descs, mps, nprob < 0 ? (int)md.size() : nprob, cp,
                                                                  ctx.d_err);
        TNS_CUDA(cudaGetLastError());
    };
    static bool configured_wide[64] = {}, configured_narrow[64] = {};
    if (trial) {
        // Both widths over the same residues; each writes the same byte planes.
        const ModDesc* nd = static_cast<const ModDesc*>(ctx.upload(md_narrow.data(), sizeof(ModDesc) * md_narrow.size()));
        const ModMaps* nmaps =
            static_cast<const ModMaps*>(ctx.upload(maps_narrow.data(), sizeof(ModMaps) * maps_narrow.size()));
        const float narrow = time_launches(ctx, [&] {
            launch(modular_gemm_kernel<128>, split_smem<128>(), configured_narrow[ctx.device], nd, nmaps, tiles_narrow);
        });
        const float wide = time_launches(ctx, [&] {
            launch(modular_gemm_kernel<256>, split_smem<256>(), configured_wide[ctx.device], d_desc, d_maps, tiles);
        });
        record_variant(ctx.device, tune_kind, tiles_wide, depth, wide <= narrow ? 1 : 0);
        ctx.autotune_trials++;
        ctx.kernel_launches++;
    } else if (tn == 256) {
        // CTA pairs over every two 128-row strips of a product; a product's
        // odd last strip by the one-CTA kernel.
        std::vector<ModDesc> pd, od;
        std::vector<ModMaps> pmaps, omaps;
        int pairs = 0, odd_tiles = 0;
        for (size_t q = 0; q < v.size(); ++q) {
            const auto& s = z[q];
            const int strips = s.mp / kTile, cols = s.np / kPairN;
            if (strips >= 2) {
                ModMaps pm;
                pm.a = maps[q].a;
                encode_residues(&pm.b, reinterpret_cast<int8_t*>(at(s.b_off)), s.kp, s.np, nm, kPairN / 2);
                pd.push_back(ModDesc{s.kp, s.np, s.mp, strips / 2, pairs, md[q].u, 0});
                pmaps.push_back(pm);
                pairs += (strips / 2) * cols;
            }
            if (strips % 2) {
                od.push_back(ModDesc{s.kp, s.np, s.mp, 1, odd_tiles, md[q].u, (strips - 1) * kTile});
                omaps.push_back(maps[q]);
                odd_tiles += cols;
            }
        }
        {
            static bool configured_pair[64] = {};
            if (!configured_pair[ctx.device]) {
                TNS_CUDA(cudaFuncSetAttribute(modular_gemm_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              kPairSmem));
                configured_pair[ctx.device] = true;
            }
            const ModDesc* pdd =
                pd.empty() ? nullptr : static_cast<const ModDesc*>(ctx.upload(pd.data(), sizeof(ModDesc) * pd.size()));
            const ModMaps* pmd = pmaps.empty() ? nullptr
                                               : static_cast<const ModMaps*>(
                                                     ctx.upload(pmaps.data(), sizeof(ModMaps) * pmaps.size()));
            const ModDesc* odd =
                od.empty() ? nullptr : static_cast<const ModDesc*>(ctx.upload(od.data(), sizeof(ModDesc) * od.size()));
            const ModMaps* omd = omaps.empty() ? nullptr
                                               : static_cast<const ModMaps*>(
                                                     ctx.upload(omaps.data(), sizeof(ModMaps) * omaps.size()));
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)(2 * pairs + odd_tiles + (odd_tiles & 1)));
            cfg.blockDim = dim3(kSplitThreads);
            cfg.dynamicSmemBytes = kPairSmem;
            cfg.stream = ctx.stream;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = 2;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            TNS_CUDA(cudaLaunchKernelEx(&cfg, modular_gemm_pair_kernel, pdd, pmd, (int)pd.size(), pairs, odd, omd,
                                        (int)od.size(), odd_tiles, cp, ctx.d_err));
        }
    } else {
        launch(modular_gemm_kernel<128>, split_smem<128>(), configured_narrow[ctx.device], d_desc, d_maps, tiles);
    }
    if (ctx.timing) {
        TNS_CUDA(cudaEventRecord(e1, ctx.stream));
        ctx.split_events.emplace_back(e0, e1);
    }
    {
        Batch<CrtDesc> b = make_batch(ctx, cd);
        crt_kernel<CPLX><<<dim3((max_out_cols + 31) / 32, (max_out_rows + 31) / 32, b.count), 256, 0, ctx.stream>>>(
            b, cp);
        TNS_CUDA(cudaGetLastError());
    }
    ctx.kernel_launches += 2;
    ctx.split_launches++;
    for (size_t q = 0; q < v.size(); ++q) {
        const auto& s = z[q];
        ctx.split_int8_ops += 2.0 * s.mp * (double)s.np * s.kp * nm;
        ctx.split_flops += (CPLX ? 8.0 : 2.0) * (double)s.m * s.n * s.k;
        ctx.split_bytes += (double)nm * ((double)s.mp * s.kp + (double)s.np * s.kp + (double)s.mp * s.np);
    }
}

}  // namespace

int split_integer_bits(int moduli, int kmax) {
    if (moduli < 8 || moduli > kMaxModuli)
        fail(TNS_E_ARGUMENT, "split-precision products take 8 to " + std::to_string(kMaxModuli) + " moduli");
    return crt_params(moduli, kmax).t;
}

void gemm_split_batch(Context& ctx, std::vector<SplitProduct>& v, int moduli) {
    std::vector<SplitProduct> live;
    for (auto& p : v) {
        if (p.a->cols != p.b->rows || p.c->rows != p.a->rows || p.c->cols != p.b->cols || p.a->cplx != p.b->cplx ||
            p.a->cplx != p.c->cplx)
            fail(TNS_E_ARGUMENT, "internal split product of non-conformable matrices");
        if (p.a->rows > 0 && p.b->cols > 0) live.push_back(p);
    }
    if (live.empty()) return;
    // Deepest products first: the modular GEMM's CTAs are dispatched in tile
    // order and a tile's time grows with its depth, so the launch ends on the
    // light tiles.
    std::stable_sort(live.begin(), live.end(),
                     [](const SplitProduct& x, const SplitProduct& y) { return x.a->cols > y.a->cols; });
    if (moduli < 8 || moduli > kMaxModuli)
        fail(TNS_E_ARGUMENT, "split-precision products take 8 to " + std::to_string(kMaxModuli) + " moduli");
    if (live[0].a->cplx) split_launch<true>(ctx, live, moduli);
    else split_launch<false>(ctx, live, moduli);
}

}  // namespace tns
