// Split-precision products: FP64 (real or complex) C := A B (+ C) computed
// from 8-bit integer slices on the tcgen05 tensor cores, with exact 32-bit
// integer accumulation and FP64 recombination (the Ozaki scheme).
//
// Slicing. Every row i of A is scaled by 2^-e_i, every column j of B by
// 2^-f_j, where 2^e bounds the row's (column's) largest magnitude from above
// (complex: the larger of |Re| and |Im|, shared by both parts), so every
// scaled entry x lies in (-1, 1). Then S signed 8-bit slices are peeled off
// exactly: x <- 128 x, a_s = trunc(x), x <- x - a_s, so that
//     A[i,k] = 2^e_i * sum_s a_s[i,k] 2^(-7 s)   (to 7 S bits of the row's scale).
// Product. The slice products with equal weight 2^(-7 d), d = s + t, are summed
// in one 32-bit integer accumulator (exact: |a_s|,|b_t| <= 127, at most S
// pairs, K' <= the limit checked on the host); pairs with d > S + 1 are left
// out, below the precision of the scheme. The FP64 result is
//     C[i,j] = 2^(e_i + f_j) * sum_{d = S+1 .. 2} 2^(-7 d) P_d[i,j],
// summed from the smallest weight to the largest.
// Complex. With the real and imaginary parts sharing their exponents, the
// complex product is the single real product
//     [Ar Ai] * [[Br, Bi], [-Bi, Br]]   (columns of the right factor interleaved,
// so that output columns 2j, 2j+1 are Re, Im of C[:, j]) -- four real
// multiplications per complex multiply-add, as the 4M method (never 3M).
//
// Kernel. One CTA per 128 x 128 output tile: a TMA producer warp streams
// 128 x 128-byte slice tiles (128-byte swizzle) through a 4-stage mbarrier
// ring; one thread issues tcgen05.mma kind::i8 (M = N = 128, K = 32) into one of
// two TMEM accumulators (columns 0..255); four epilogue warps read each
// finished accumulator (tcgen05.ld), add its weighted FP64 value into a
// running FP64 sum kept in TMEM (columns 256..511, two per double) and, after
// the last weight, scale and store C. The epilogue of one weight overlaps
// the MMAs of the next. Every wait is bounded; TMEM is released on every path.
//
// Accuracy: the result differs from an FP64 product by at most about
// K 2^(-7 S) (row scale)(column scale) per entry; with S = 8 that is at the
// level of FP64 rounding for the orders used here. It does not reproduce the
// reference's rounding order; it is the split-precision form of the product.

#include "batch.cuh"
#include "device_util.cuh"
#include "tcgen05.cuh"
#include "tns_internal.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <string>
#include <vector>

namespace tns {

namespace {

constexpr int kTile = 128;       // output tile rows and columns; slice tile rows
constexpr int kKb = 128;         // bytes (8-bit elements) of K per stage
constexpr int kStages = 4;
constexpr uint32_t kStageBytes = 2u * kTile * kKb;  // A and B tiles, 16 KB each
constexpr int kSplitThreads = 192;                  // producer, MMA, 4 epilogue warps
constexpr uint32_t kTmemCols = 512;                 // 2 x 128 accumulators + 128 doubles
constexpr int kSplitSmem = kStages * (int)kStageBytes + 1024 + 256;

enum : int { kErrSplitFull = 11, kErrSplitEmpty = 12, kErrSplitAcc = 13, kErrSplitDrain = 14 };

// ---- exponents ---------------------------------------------------------------

// 2^e with e the least integer such that every |x| < 2^e (0 for an all-zero set).
__device__ __forceinline__ int bound_exponent(double m) { return m > 0.0 ? ilogb(m) + 1 : 0; }

struct ExpDesc {
    const double* a;  // column-major, ld elements
    int ld, rows, cols;
    int* out;
};

// Row exponents of A: one thread per row, over every column.
template <bool CPLX>
__global__ void row_exponent_kernel(const __grid_constant__ Batch<ExpDesc> b) {
    const ExpDesc& d = batch_item(b, blockIdx.y);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.rows) return;
    double m = 0.0;
    for (int k = 0; k < d.cols; ++k) {
        if (CPLX) {
            const double2 z = reinterpret_cast<const double2*>(d.a)[(size_t)k * d.ld + i];
            m = fmax(m, fmax(fabs(z.x), fabs(z.y)));
        } else {
            m = fmax(m, fabs(d.a[(size_t)k * d.ld + i]));
        }
    }
    d.out[i] = bound_exponent(m);
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

// ---- slicing ---------------------------------------------------------------------

// Peels S signed 8-bit slices off x in (-1, 1); exact.
template <int S>
__device__ __forceinline__ void peel(double x, int8_t (&a)[S]) {
#pragma unroll
    for (int s = 0; s < S; ++s) {
        x *= 128.0;
        const double t = trunc(x);
        x -= t;
        a[s] = (int8_t)(int)t;
    }
}

struct SliceDesc {
    const double* src;  // A (rows x k) or B (k x cols), column-major, ld elements
    int ld, m, k;       // logical rows (A) or columns (B); depth
    int rows_p, kp;     // padded slice extents: rows of the slice array, bytes per row
    const int* e;       // exponents of the rows (A) or columns (B)
    int8_t* dst;        // S x rows_p x kp
};

// A': row i holds [Re A(i,:), Im A(i,:)] (real: A(i,:)), 16 bytes per thread.
template <bool CPLX, int S>
__global__ void slice_a_kernel(const __grid_constant__ Batch<SliceDesc> b) {
    const SliceDesc& d = batch_item(b, blockIdx.z);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int c0 = blockIdx.y * 16;
    if (i >= d.rows_p || c0 >= d.kp) return;
    const int e = i < d.m ? d.e[i] : 0;
    alignas(16) int8_t out[S][16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int kk = c0 + u;
        double v = 0.0;
        if (i < d.m) {
            if (CPLX) {
                if (kk < d.k) v = d.src[((size_t)kk * d.ld + i) * 2];
                else if (kk < 2 * d.k) v = d.src[((size_t)(kk - d.k) * d.ld + i) * 2 + 1];
            } else if (kk < d.k) {
                v = d.src[(size_t)kk * d.ld + i];
            }
        }
        int8_t a[S];
        peel<S>(scalbn(v, -e), a);
#pragma unroll
        for (int s = 0; s < S; ++s) out[s][u] = a[s];
    }
#pragma unroll
    for (int s = 0; s < S; ++s)
        *reinterpret_cast<int4*>(d.dst + ((size_t)s * d.rows_p + i) * d.kp + c0) = *reinterpret_cast<int4*>(out[s]);
}

// B': row n of the right factor, K-major. Complex: row 2j = [Re B(:,j); -Im B(:,j)],
// row 2j+1 = [Im B(:,j); Re B(:,j)]; real: row j = B(:,j). 16 bytes per thread.
template <bool CPLX, int S>
__global__ void slice_b_kernel(const __grid_constant__ Batch<SliceDesc> b) {
    const SliceDesc& d = batch_item(b, blockIdx.y);
    const int chunks = d.kp / 16;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)chunks * d.rows_p) return;
    const int n = (int)(idx / chunks), c0 = (int)(idx % chunks) * 16;
    const int j = CPLX ? n / 2 : n;
    const bool live = j < d.m;
    const int e = live ? d.e[j] : 0;
    alignas(16) int8_t out[S][16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int kk = c0 + u;
        double v = 0.0;
        if (live) {
            if (CPLX) {
                const bool top = kk < d.k;
                const int k = top ? kk : kk - d.k;
                if (kk < 2 * d.k) {
                    const double2 z = reinterpret_cast<const double2*>(d.src)[(size_t)j * d.ld + k];
                    // even rows: (Re; -Im), odd rows: (Im; Re)
                    v = (n & 1) ? (top ? z.y : z.x) : (top ? z.x : -z.y);
                }
            } else if (kk < d.k) {
                v = d.src[(size_t)j * d.ld + kk];
            }
        }
        int8_t a[S];
        peel<S>(scalbn(v, -e), a);
#pragma unroll
        for (int s = 0; s < S; ++s) out[s][u] = a[s];
    }
#pragma unroll
    for (int s = 0; s < S; ++s)
        *reinterpret_cast<int4*>(d.dst + ((size_t)s * d.rows_p + n) * d.kp + c0) = *reinterpret_cast<int4*>(out[s]);
}

// ---- the product --------------------------------------------------------------------

struct SplitDesc {
    int m, n;                // output rows and (complex or real) columns
    int kp;                  // bytes per slice row (multiple of 128)
    int tiles_m, tile_begin;
    const int* ea;           // row exponents of A
    const int* eb;           // column exponents of B
    double* c;               // column-major output (complex interleaved), ld elements
    int ldc;
    int accumulate;          // 0: C = AB, 1: C += AB
};
struct SplitMaps {
    CUtensorMap a, b;  // slices as (kp bytes) x (rows) x S, boxes of 128 x 128 x 1, 128-byte swizzle
};

template <bool CPLX, int S>
__global__ void __launch_bounds__(kSplitThreads, 1)
    split_gemm_kernel(const SplitDesc* __restrict__ descs, const SplitMaps* __restrict__ maps, int nprob, int* err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
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
        if (descs[mid].tile_begin <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const SplitDesc& D = descs[lo];
    const SplitMaps& MP = maps[lo];
    const int local = blockIdx.x - D.tile_begin;
    const int m0 = (local % D.tiles_m) * kTile, n0 = (local / D.tiles_m) * kTile;
    const int nkb = D.kp / kKb;

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
            for (int q = 0; q < S && ok; ++q) {
                const int dsum = S + 1 - q;
                for (int s = max(1, dsum - S); s <= min(S, dsum - 1) && ok; ++s) {
                    const int t = dsum - s;
                    for (int kb = 0; kb < nkb; ++kb) {
                        const int st = issued % kStages;
                        if (!mbar_wait_bounded(&empty[st], ((issued / kStages) & 1) ^ 1, err, kErrSplitEmpty)) {
                            ok = false;
                            break;
                        }
                        mbar_arrive_expect_tx(&full[st], kStageBytes);
                        tma_load_3d(stage_a(st), &MP.a, kb * kKb, m0, s - 1, &full[st]);
                        tma_load_3d(stage_b(st), &MP.b, kb * kKb, n0, t - 1, &full[st]);
                        ++issued;
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = i8_instr_desc(kTile, kTile);
            uint32_t it = 0;
            bool ok = true;
            for (int q = 0; q < S && ok; ++q) {
                const int dsum = S + 1 - q, buf = q & 1;
                if (!mbar_wait_bounded(&acce[buf], ((q >> 1) & 1) ^ 1, err, kErrSplitAcc)) break;
                tc_fence_after_sync();
                const uint32_t dacc = tmem + buf * kTile;
                bool first = true;
                for (int s = max(1, dsum - S); s <= min(S, dsum - 1) && ok; ++s) {
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
                                   idesc, !(first && kk == 0));
                        }
                        first = false;
                        mma_commit(&empty[st]);
                        ++it;
                    }
                }
                if (ok) mma_commit(&accf[buf]);
            }
            *consumed = it;
            mma_commit(done);
        }
    } else {
        // Epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (the rows of the tile).
        const int quarter = warp & 3;
        const int row = quarter * 32 + lane;
        const int i = m0 + row;
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        const int ei = i < D.m ? D.ea[i] : 0;
        for (int q = 0; q < S; ++q) {
            const int dsum = S + 1 - q, buf = q & 1;
            // The TMEM moves below are warp-collective: the warp goes on only
            // if every lane saw the accumulator complete.
            const bool got = mbar_wait_bounded(&accf[buf], (q >> 1) & 1, err, kErrSplitAcc);
            if (!__all_sync(0xffffffffu, got)) break;
            tc_fence_after_sync();
            const double w = scalbn(1.0, -7 * dsum);
            for (int c0 = 0; c0 < kTile; c0 += 16) {
                uint32_t v[16], f0[16], f1[16];
                tmem_ld16(tmem + lane_addr + buf * kTile + c0, v);
                if (q > 0) {
                    tmem_ld16(tmem + lane_addr + 2 * kTile + 2 * c0, f0);
                    tmem_ld16(tmem + lane_addr + 2 * kTile + 2 * c0 + 16, f1);
                }
                tmem_wait_ld();
                double acc[16];
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const double x = (double)(int)v[e] * w;
                    if (q > 0) {
                        const uint32_t* f = e < 8 ? f0 : f1;
                        const int o = (e & 7) * 2;
                        acc[e] = __hiloint2double((int)f[o + 1], (int)f[o]) + x;
                    } else {
                        acc[e] = x;
                    }
                }
                if (q < S - 1) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        uint32_t* f = e < 8 ? f0 : f1;
                        const int o = (e & 7) * 2;
                        f[o] = (uint32_t)__double2loint(acc[e]);
                        f[o + 1] = (uint32_t)__double2hiint(acc[e]);
                    }
                    tmem_st16(tmem + lane_addr + 2 * kTile + 2 * c0, f0);
                    tmem_st16(tmem + lane_addr + 2 * kTile + 2 * c0 + 16, f1);
                } else if (i < D.m) {
                    if (CPLX) {
#pragma unroll
                        for (int e = 0; e < 16; e += 2) {
                            const int j = (n0 + c0 + e) >> 1;
                            if (j >= D.n) continue;
                            const int sc = ei + D.eb[j];
                            double2 r = make_double2(scalbn(acc[e], sc), scalbn(acc[e + 1], sc));
                            double2* p = reinterpret_cast<double2*>(D.c) + (size_t)j * D.ldc + i;
                            if (D.accumulate) {
                                const double2 o = *p;
                                r = make_double2(o.x + r.x, o.y + r.y);
                            }
                            *p = r;
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const int j = n0 + c0 + e;
                            if (j >= D.n) continue;
                            double r = scalbn(acc[e], ei + D.eb[j]);
                            double* p = D.c + (size_t)j * D.ldc + i;
                            if (D.accumulate) r += *p;
                            *p = r;
                        }
                    }
                }
            }
            if (q < S - 1) tmem_wait_st();
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

// The slices of one operand as a 3-D byte array (kp x rows_p x S), boxes of
// 128 x 128 x 1 with 128-byte swizzle.
void encode_slices(CUtensorMap* map, const int8_t* base, int kp, int rows_p, int S) {
    cuuint64_t dims[3] = {(cuuint64_t)kp, (cuuint64_t)rows_p, (cuuint64_t)S};
    cuuint64_t strides[2] = {(cuuint64_t)kp, (cuuint64_t)kp * rows_p};
    cuuint32_t box[3] = {(cuuint32_t)kKb, (cuuint32_t)kTile, 1};
    cuuint32_t elem[3] = {1, 1, 1};
    CUresult r = tensor_map_encoder()(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t*>(base), dims, strides,
                                      box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        fail(TNS_E_DEVICE, "TMA descriptor encoding for the split product failed (CUresult " + std::to_string((int)r) + ")");
}

template <bool CPLX, int S>
void split_launch(Context& ctx, std::vector<SplitProduct>& v) {
    constexpr int DPE = CPLX ? 2 : 1;
    struct Sizes {
        int m, n, k, mp, np, kp;
        size_t a_off, b_off, ea_off, eb_off;
    };
    std::vector<Sizes> z;
    size_t total = 0;
    auto take = [&](size_t bytes) {
        size_t off = total;
        total += (bytes + 255) & ~size_t(255);
        return off;
    };
    for (auto& p : v) {
        Sizes s{};
        s.m = p.a->rows;
        s.k = p.a->cols;
        s.n = p.b->cols;
        s.mp = round_up(s.m, kTile);
        s.np = round_up(DPE * s.n, kTile);
        s.kp = round_up(DPE * s.k, kKb);
        // Exactness of the 32-bit sums: at most S pairs of K' products of |127|^2.
        if ((double)S * s.kp * 127.0 * 127.0 >= 2147483647.0)
            fail(TNS_E_ARGUMENT, "split-precision product too deep for exact 32-bit accumulation");
        s.a_off = take((size_t)S * s.mp * s.kp);
        s.b_off = take((size_t)S * s.np * s.kp);
        s.ea_off = take(sizeof(int) * s.mp);
        s.eb_off = take(sizeof(int) * std::max(1, s.n));
        z.push_back(s);
    }
    DBuf scratch(ctx, total);
    auto at = [&](size_t off) { return static_cast<char*>(scratch.p) + off; };

    std::vector<ExpDesc> rows, cols;
    std::vector<SliceDesc> sa, sb;
    std::vector<SplitDesc> gd;
    std::vector<SplitMaps> maps(v.size());
    int max_m = 0, max_cols = 0, max_rows_a = 0, max_chunks = 0;
    long long max_b_threads = 0;
    int tiles = 0;
    for (size_t q = 0; q < v.size(); ++q) {
        const auto& p = v[q];
        const auto& s = z[q];
        int* ea = reinterpret_cast<int*>(at(s.ea_off));
        int* eb = reinterpret_cast<int*>(at(s.eb_off));
        int8_t* a8 = reinterpret_cast<int8_t*>(at(s.a_off));
        int8_t* b8 = reinterpret_cast<int8_t*>(at(s.b_off));
        rows.push_back(ExpDesc{p.a->p, p.a->ld(), s.m, s.k, ea});
        cols.push_back(ExpDesc{p.b->p, p.b->ld(), s.k, s.n, eb});
        sa.push_back(SliceDesc{p.a->p, p.a->ld(), s.m, s.k, s.mp, s.kp, ea, a8});
        sb.push_back(SliceDesc{p.b->p, p.b->ld(), s.n, s.k, s.np, s.kp, eb, b8});
        SplitDesc g{};
        g.m = s.m;
        g.n = s.n;
        g.kp = s.kp;
        g.tiles_m = s.mp / kTile;
        g.tile_begin = tiles;
        g.ea = ea;
        g.eb = eb;
        g.c = p.c->p;
        g.ldc = p.c->ld();
        g.accumulate = p.beta != 0.0 ? 1 : 0;
        gd.push_back(g);
        tiles += (s.mp / kTile) * (s.np / kTile);
        encode_slices(&maps[q].a, a8, s.kp, s.mp, S);
        encode_slices(&maps[q].b, b8, s.kp, s.np, S);
        max_m = std::max(max_m, s.m);
        max_cols = std::max(max_cols, s.n);
        max_rows_a = std::max(max_rows_a, s.mp);
        max_chunks = std::max(max_chunks, s.kp / 16);
        max_b_threads = std::max(max_b_threads, (long long)(s.kp / 16) * s.np);
    }
    if (tiles == 0) return;
    {
        Batch<ExpDesc> br = make_batch(ctx, rows);
        row_exponent_kernel<CPLX><<<dim3((max_m + 127) / 128, br.count), 128, 0, ctx.stream>>>(br);
        TNS_CUDA(cudaGetLastError());
        Batch<ExpDesc> bc = make_batch(ctx, cols);
        col_exponent_kernel<CPLX><<<dim3((max_cols + 7) / 8, bc.count), 256, 0, ctx.stream>>>(bc);
        TNS_CUDA(cudaGetLastError());
        Batch<SliceDesc> bsa = make_batch(ctx, sa);
        slice_a_kernel<CPLX, S><<<dim3((max_rows_a + 127) / 128, max_chunks, bsa.count), 128, 0, ctx.stream>>>(bsa);
        TNS_CUDA(cudaGetLastError());
        Batch<SliceDesc> bsb = make_batch(ctx, sb);
        slice_b_kernel<CPLX, S><<<dim3((unsigned)((max_b_threads + 127) / 128), bsb.count), 128, 0, ctx.stream>>>(bsb);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches += 4;
    }
    static bool configured[64] = {};
    if (!configured[ctx.device]) {
        TNS_CUDA(cudaFuncSetAttribute(split_gemm_kernel<CPLX, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      kSplitSmem));
        configured[ctx.device] = true;
    }
    const SplitDesc* d_desc = static_cast<const SplitDesc*>(ctx.upload(gd.data(), sizeof(SplitDesc) * gd.size()));
    const SplitMaps* d_maps = static_cast<const SplitMaps*>(ctx.upload(maps.data(), sizeof(SplitMaps) * maps.size()));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ctx.timing) {
        e0 = ctx.take_event();
        e1 = ctx.take_event();
        TNS_CUDA(cudaEventRecord(e0, ctx.stream));
    }
    split_gemm_kernel<CPLX, S><<<tiles, kSplitThreads, kSplitSmem, ctx.stream>>>(d_desc, d_maps, (int)gd.size(),
                                                                                 ctx.d_err);
    TNS_CUDA(cudaGetLastError());
    if (ctx.timing) {
        TNS_CUDA(cudaEventRecord(e1, ctx.stream));
        ctx.split_events.emplace_back(e0, e1);
    }
    ctx.kernel_launches++;
    ctx.split_launches++;
    for (size_t q = 0; q < v.size(); ++q) {
        const auto& s = z[q];
        const int pairs = S * (S + 1) / 2;
        ctx.split_int8_ops += 2.0 * s.mp * (double)s.np * s.kp * pairs;
        ctx.split_flops += (CPLX ? 8.0 : 2.0) * (double)s.m * s.n * s.k;
    }
}

}  // namespace

void gemm_split_batch(Context& ctx, std::vector<SplitProduct>& v, int slices) {
    std::vector<SplitProduct> live;
    for (auto& p : v) {
        if (p.a->cols != p.b->rows || p.c->rows != p.a->rows || p.c->cols != p.b->cols || p.a->cplx != p.b->cplx ||
            p.a->cplx != p.c->cplx)
            fail(TNS_E_ARGUMENT, "internal split product of non-conformable matrices");
        if (p.a->rows > 0 && p.b->cols > 0) live.push_back(p);
    }
    if (live.empty()) return;
    const bool cplx = live[0].a->cplx;
#define TNS_SPLIT(SV)                                              \
    case SV:                                                       \
        if (cplx) split_launch<true, SV>(ctx, live);               \
        else split_launch<false, SV>(ctx, live);                   \
        return;
    switch (slices) {
        TNS_SPLIT(4)
        TNS_SPLIT(5)
        TNS_SPLIT(6)
        TNS_SPLIT(7)
        TNS_SPLIT(8)
        default: fail(TNS_E_ARGUMENT, "split-precision products take 4 to 8 slices");
    }
#undef TNS_SPLIT
}

}  // namespace tns
