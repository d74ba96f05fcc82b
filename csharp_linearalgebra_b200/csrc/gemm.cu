// FP64 GEMM on the B200 tensor cores (DMMA), real and complex (4M).
//
// Replaces the reference's BLIS-style CPU GEMM (src/Tensile.Kernels/Gemm.cs:117-203,
// ParallelGemm.cs:138-229, MicroKernels.cs:57-273) and its 4M complex product
// (src/Tensile/ComplexKernels.cs:49-108). C := beta*C + alpha*A*B, column-major.
//
// Design
//  - tcgen05 has no f64 kind, so the math is warp-level mma.sync m16n8k4 f64.
//    Measured on B200, a DMMA accumulation is bit-identical to a chain of
//    fused multiply-adds in k order -- the reference micro-kernel's inner loop
//    -- so the kernel reproduces the reference's result bit for bit by folding
//    the accumulator into C (c = fma(alpha, acc, c)) at the end of each
//    KC-deep slab, where the reference writes back, with the reference's KC.
//  - Complex products keep the reference's 4M order: pass 1 forms
//    P = Ar*Br and Q = Ar*Bi slab by slab, pass 2 folds in P -= Ai*Bi and
//    Q += Ai*Br, then P + iQ is combined into C with the reference's alpha and
//    beta special cases (ComplexKernels.Combine). Both passes stream the same
//    interleaved tiles; no split copies of A or B are made.
//  - Operand tiles are staged in shared memory by tiled TMA loads
//    (cp.async.bulk.tensor.2d; one box of B and one or two of A per k-step)
//    completing on mbarriers; a producer warp runs STAGES k-steps ahead of the
//    math warps. Each box is loaded wider than its tile so that its columns
//    land padded and the DMMA fragment loads are bank-conflict free (real: A
//    stride = 4 mod 16 doubles, B stride 20; complex: A stride = 2 mod 8
//    complex, B stride 20). The extra rows are real data or the TMA unit's
//    zero fill beyond the operand, and are never multiplied.
//  - The MMA computes C^T = B^T A^T, so a thread's accumulator pair covers two
//    consecutive rows of column-major C and the epilogue moves 16-byte pairs.
//  - Persistent CTAs walk a list of problems (grouped GEMM): the same kernel
//    serves one product, or every matrix of a batch in one launch.
//  - A single product with fewer tiles than SMs and several KC slabs (1024^3:
//    64 tiles of 128 x 128, four slabs) is slab-split: every (tile, slab,
//    pass) is a unit of its own, writes its raw slab product to a plane, and
//    a fold kernel adds the planes into C in slab order. Each slab's
//    accumulation starts from zero in both forms, so the split changes which
//    CTA computes a slab, not the operations, and C gets the same bits.
//  - Every wait is bounded (device_util.cuh): a stuck pipeline records an error
//    in the context flag and the kernel returns.
//
// Operand requirements (checked on the host before every launch): pointers and
// leading dimensions 16-byte aligned, M and N even, K and KC multiples of 16.
// The library's device matrices are zero-padded to multiples of 64, which
// meets all of them.

#include "device_util.cuh"
#include "tns_internal.h"
#include "autotune.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <string>
#include <type_traits>
#include <vector>

namespace tns {

template <bool CPLX, int WARPS_M, int WARPS_N, int STAGES_>
struct GemmCfg {
    static constexpr bool kComplex = CPLX;
    static constexpr int ESZ = CPLX ? 16 : 8;  // bytes per element
    static constexpr int WM = 32;              // C rows per warp = 4 mma-N fragments of 8
    static constexpr int WN = CPLX ? 32 : 64;  // C columns per warp, mma-M fragments of 16
    static constexpr int MF = WM / 8;
    static constexpr int NF = WN / 16;
    static constexpr int BM = WARPS_M * WM;
    static constexpr int BN = WARPS_N * WN;
    static constexpr int BK = 16;
    static constexpr int STAGES = STAGES_;
    // A stage holds A_BOXES TMA boxes of A_BOX_ROWS rows (complex boxes stop
    // at 64 rows: a box row may hold at most 256 doubles). Each box is loaded
    // wider than its rows, so its columns land padded in shared memory.
    static constexpr int A_BOX_ROWS = CPLX ? 64 : BM;
    static constexpr int A_BOXES = BM / A_BOX_ROWS;
    static constexpr int LDA_S = A_BOX_ROWS + (CPLX ? 2 : 4);  // smem A column stride, elements
    static constexpr int LDB_S = BK + 4;                       // smem B column stride, elements
    static constexpr int A_BOX = BK * LDA_S;                   // elements
    static constexpr int A_STAGE = A_BOXES * A_BOX;
    static constexpr int B_STAGE = BN * LDB_S;
    static constexpr int DPE = CPLX ? 2 : 1;  // doubles per element (TMA maps count doubles)
    static constexpr int STAGE_BYTES = (A_STAGE + B_STAGE) * ESZ;
    static constexpr int CONSUMERS = WARPS_M * WARPS_N;
    // Eight math warps plus one producer warp would put three warps on one SM
    // sub-partition and cap every thread at 168 registers. Instead the
    // producer is a whole warpgroup (one warp feeds, three leave) that hands
    // registers to the math warpgroups: launched at 168 per thread,
    // 128 x 40 + 256 x 232 = 384 x 168, the launch's whole allocation.
    static constexpr bool kSplitRegs = CONSUMERS == 8;
    static constexpr int kLaunchRegs = 168, kProducerRegs = 40, kMathRegs = 232;
    static_assert(!kSplitRegs || 128 * kProducerRegs + 256 * kMathRegs == 384 * kLaunchRegs, "register split");
    static constexpr int THREADS = (CONSUMERS + (kSplitRegs ? 4 : 1)) * 32;
    // stages, full and empty barriers, the tile announced with each stage, alignment slack
    static constexpr int SMEM = STAGES * STAGE_BYTES + 2 * STAGES * 8 + STAGES * 4 + 128;
    static_assert((LDA_S * ESZ) % 16 == 0 && (LDB_S * ESZ) % 16 == 0, "smem columns must stay 16B aligned");
    static_assert((A_BOX * ESZ) % 128 == 0 && (B_STAGE * ESZ) % 128 == 0, "TMA boxes land 128B aligned");
    static_assert(LDA_S * DPE <= 256 && LDB_S * DPE <= 256 && BN <= 256, "TMA box extents");
    static_assert(WM <= A_BOX_ROWS && A_BOX_ROWS % WM == 0, "a warp's rows stay inside one A box");
    static_assert(SMEM <= 227 * 1024, "shared memory budget");
};

__device__ __forceinline__ int find_problem(const GemmProblem* probs, int nprob, int tile) {
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (probs[mid].tile_begin <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The TMA descriptors of one problem's operands, viewed as 2-D arrays of
// doubles (complex: two doubles per element): A is (DPE*M) x K, B is
// (DPE*K) x N, column-major with the problem's leading dimensions.
struct GemmMaps {
    CUtensorMap a, b;
};

// Problems of one launch: up to four travel in the parameter block with their
// descriptors, a longer list (and its descriptors) lives in device memory.
struct GemmLaunch {
    GemmProblem inl[4];
    GemmMaps inl_maps[4];
    const GemmProblem* list;
    const GemmMaps* maps_list;
    unsigned long long* tiles;  // zeroed tile counter (dynamic order), or null (static round robin)
    int nprob;
    int total_tiles;
    int* err;
};

// Combine (ComplexKernels.cs:213-240): alpha (P + iQ) + beta C with the
// reference's special cases for unit and real alpha, zero and unit beta. C is
// read only when beta is nonzero.
__device__ __forceinline__ double2 combine_4m(double2 pq, double ar, double ai, double br, double bi,
                                              const double2* c_at) {
    const bool unit_alpha = (ar == 1.0 && ai == 0.0);
    const bool real_alpha = (ai == 0.0);
    const bool zero_beta = (br == 0.0 && bi == 0.0);
    const bool unit_beta = (br == 1.0 && bi == 0.0);
    double pr, pi;
    if (unit_alpha) {
        pr = pq.x;
        pi = pq.y;
    } else if (real_alpha) {
        pr = mul_rn(ar, pq.x);
        pi = mul_rn(ar, pq.y);
    } else {
        pr = sub_rn(mul_rn(ar, pq.x), mul_rn(ai, pq.y));
        pi = add_rn(mul_rn(ai, pq.x), mul_rn(ar, pq.y));
    }
    if (zero_beta) return make_double2(pr, pi);
    const double2 c = *c_at;
    if (unit_beta) return make_double2(add_rn(c.x, pr), add_rn(c.y, pi));
    const double cr = sub_rn(mul_rn(br, c.x), mul_rn(bi, c.y));
    const double ci = add_rn(mul_rn(bi, c.x), mul_rn(br, c.y));
    return make_double2(add_rn(cr, pr), add_rn(ci, pi));
}

// The k-range of one unit of work. Unsplit, a unit is a tile: all of K, every
// pass. Slab-split (SPLIT), a unit is one tile's one KC slab of one pass, and
// the units of a problem are numbered pass-major, then slab, then tile.
struct UnitRange {
    int local;  // the tile within its problem
    int part;   // pass * slabs + slab (slab-split), else 0
    int kt0;    // first k-step
    int iters;  // k-steps the unit runs (all passes' when unsplit)
};

template <bool SPLIT, int PASSES>
__device__ __forceinline__ UnitRange unit_range(const GemmProblem& P, int local, int bk) {
    const int nk = P.K / bk;
    UnitRange u{local, 0, 0, nk * PASSES};
    if constexpr (SPLIT) {
        const int tiles = P.tiles_m * P.tiles_n;
        const int slab_kt = P.kc / bk;
        u.part = local / tiles;
        u.local = local - u.part * tiles;
        u.kt0 = (u.part % P.slabs) * slab_kt;
        u.iters = min(nk - u.kt0, slab_kt);
    }
    return u;
}

template <class Cfg, bool SPLIT>
__global__ void __launch_bounds__(Cfg::THREADS, 1) gemm_dmma_kernel(const __grid_constant__ GemmLaunch L) {
    using E = typename std::conditional<Cfg::kComplex, double2, double>::type;
    constexpr int PASSES = Cfg::kComplex ? 2 : 1;
    const GemmProblem* probs = L.list ? L.list : L.inl;
    const int nprob = L.nprob;
    const int total_tiles = L.total_tiles;
    int* err = L.err;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + Cfg::STAGES * Cfg::STAGE_BYTES);
    uint64_t* empty = full + Cfg::STAGES;
    // The producer writes the tile a stage starts (or -1: no more tiles)
    // before the stage's arrival, which releases it to the math warps.
    int* tile_slot = reinterpret_cast<int*>(empty + Cfg::STAGES);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < Cfg::STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], Cfg::CONSUMERS);
        }
        mbar_fence_init();
    }
    __syncthreads();

    auto stage_a = [&](int s) { return reinterpret_cast<E*>(smem + s * Cfg::STAGE_BYTES); };
    auto stage_b = [&](int s) {
        return reinterpret_cast<E*>(smem + s * Cfg::STAGE_BYTES + Cfg::A_STAGE * Cfg::ESZ);
    };

    if constexpr (Cfg::kSplitRegs) {
        if (warp >= Cfg::CONSUMERS) {
            reg_dealloc<Cfg::kProducerRegs>();
            if (warp != Cfg::CONSUMERS) return;  // only the warpgroup's first warp feeds
        } else {
            reg_alloc<Cfg::kMathRegs>();
        }
    }

    if (warp == Cfg::CONSUMERS) {
        // ------------------------------ producer ------------------------------
        // One lane issues each stage as A_BOXES + 1 tiled TMA loads. Boxes
        // reaching past the operand's extent are zero-filled by the TMA unit,
        // so every stage carries exactly STAGE_BYTES.
        const GemmMaps* maps = L.maps_list ? L.maps_list : L.inl_maps;
        uint32_t it = 0;
        bool ok = true;
        // Tiles in the order of the launch's list: taken from the shared
        // counter as the CTA frees up (the host lists the heaviest problems
        // first), or round robin without one.
        long long taken = 0;
        auto next_tile = [&]() -> int {
            int t = -1;
            if (lane == 0) {
                const unsigned long long v = L.tiles ? atomicAdd(L.tiles, 1ull)
                                                     : (unsigned long long)blockIdx.x + taken * gridDim.x;
                t = v < (unsigned long long)total_tiles ? (int)v : -1;
            }
            ++taken;
            return __shfl_sync(0xffffffffu, t, 0);
        };
        while (ok) {
            const int tile = next_tile();
            if (tile < 0) {
                // End marker: a stage without copies announcing no tile.
                const int s = it % Cfg::STAGES;
                if (!mbar_wait_bounded(&empty[s], ((it / Cfg::STAGES) & 1) ^ 1, err, kDevTimeoutEmpty)) {
                    ok = false;
                    break;
                }
                if (lane == 0) {
                    tile_slot[s] = -1;
                    mbar_arrive(&full[s]);
                }
                __syncwarp();
                break;
            }
            const int pi = find_problem(probs, nprob, tile);
            const GemmProblem& P = probs[pi];
            const CUtensorMap* ma = &maps[pi].a;
            const CUtensorMap* mb = &maps[pi].b;
            if (L.maps_list && lane == 0) {
                tensormap_acquire(ma);
                tensormap_acquire(mb);
            }
            const UnitRange u = unit_range<SPLIT, PASSES>(P, tile - P.tile_begin, Cfg::BK);
            int m0 = (u.local % P.tiles_m) * Cfg::BM;
            int n0 = (u.local / P.tiles_m) * Cfg::BN;
            const int nk = P.K / Cfg::BK;
            for (int q = 0; q < u.iters; ++q, ++it) {
                const int k0 = (SPLIT ? u.kt0 + q : q % nk) * Cfg::BK;
                int s = it % Cfg::STAGES;
                uint32_t round = it / Cfg::STAGES;
                if (!mbar_wait_bounded(&empty[s], (round & 1) ^ 1, err, kDevTimeoutEmpty)) {
                    ok = false;
                    break;
                }
                if (lane == 0) {
                    if (q == 0) tile_slot[s] = tile;
                    mbar_arrive_expect_tx(&full[s], (uint32_t)Cfg::STAGE_BYTES);
                    E* As = stage_a(s);
#pragma unroll
                    for (int h = 0; h < Cfg::A_BOXES; ++h)
                        tma_load_2d(As + h * Cfg::A_BOX, ma, Cfg::DPE * (m0 + h * Cfg::A_BOX_ROWS), k0, &full[s]);
                    tma_load_2d(stage_b(s), mb, Cfg::DPE * k0, n0, &full[s]);
                }
                __syncwarp();
            }
        }
        // Drain: do not leave while copies into this CTA's shared memory are in
        // flight. The consumers release every stage they read, so waiting for
        // the last STAGES releases covers every copy issued.
        if (ok) {
            for (int r = 0; r < Cfg::STAGES && (uint32_t)r < it; ++r) {
                uint32_t j = it - 1 - r;
                int s = j % Cfg::STAGES;
                if (!mbar_wait_bounded(&empty[s], (j / Cfg::STAGES) & 1, err, kDevTimeoutDrain)) break;
            }
        }
        return;
    }

    // ------------------------------- consumers -------------------------------
    const int wm = warp % (Cfg::BM / Cfg::WM);
    const int wn = warp / (Cfg::BM / Cfg::WM);
    const int g = lane >> 2;
    const int t = lane & 3;
    uint32_t it = 0;

    for (;;) {
        // The first stage of each tile announces it (or the end).
        if (!mbar_wait_bounded(&full[it % Cfg::STAGES], (it / Cfg::STAGES) & 1, err, kDevTimeoutFull)) return;
        const int tile = tile_slot[it % Cfg::STAGES];
        if (tile < 0) break;
        const GemmProblem& P = probs[find_problem(probs, nprob, tile)];
        const UnitRange u = unit_range<SPLIT, PASSES>(P, tile - P.tile_begin, Cfg::BK);
        const int m0 = (u.local % P.tiles_m) * Cfg::BM;
        const int n0 = (u.local / P.tiles_m) * Cfg::BN;
        const int nk = P.K / Cfg::BK;
        const int slab = P.kc / Cfg::BK;  // k-tiles per KC slab
        const double ar = P.alpha_re, ai = P.alpha_im, br = P.beta_re, bi = P.beta_im;

        // acc0: real part / P-pass product, acc1 (complex): Q-pass product
        double acc0[Cfg::NF][Cfg::MF][4];
        double acc1[Cfg::kComplex ? Cfg::NF : 1][Cfg::kComplex ? Cfg::MF : 1][4];
        auto zero_acc = [&]() {
#pragma unroll
            for (int i = 0; i < Cfg::NF; ++i)
#pragma unroll
                for (int j = 0; j < Cfg::MF; ++j)
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        acc0[i][j][r] = 0.0;
                        if constexpr (Cfg::kComplex) acc1[i][j][r] = 0.0;
                    }
        };
        zero_acc();

        for (int q = 0; q < u.iters; ++q, ++it) {
            const int pass = SPLIT ? u.part / P.slabs : q / nk;
            const int kt = SPLIT ? u.kt0 + q : q % nk;
            int s = it % Cfg::STAGES;
            if (q > 0 && !mbar_wait_bounded(&full[s], (it / Cfg::STAGES) & 1, err, kDevTimeoutFull)) return;
            const E* As = stage_a(s) + (wm * Cfg::WM / Cfg::A_BOX_ROWS) * Cfg::A_BOX +
                          (wm * Cfg::WM) % Cfg::A_BOX_ROWS + g;
            const E* Bs = stage_b(s) + (wn * Cfg::WN + g) * Cfg::LDB_S + t;
            // One k-step of DMMAs; PASS selects the half of A (complex) the
            // pass multiplies, so each pass loads only that half.
            auto mma_step = [&](auto pass_tag) {
                constexpr int PASS = decltype(pass_tag)::value;
                const double* Ad = reinterpret_cast<const double*>(As);
#pragma unroll
                for (int ks = 0; ks < Cfg::BK; ks += 4) {
                    E fa0[Cfg::NF], fa1[Cfg::NF];
                    double fb[Cfg::MF];
#pragma unroll
                    for (int i = 0; i < Cfg::NF; ++i) {
                        fa0[i] = Bs[(i * 16) * Cfg::LDB_S + ks];
                        fa1[i] = Bs[(i * 16 + 8) * Cfg::LDB_S + ks];
                    }
#pragma unroll
                    for (int j = 0; j < Cfg::MF; ++j) {
                        const int e = (ks + t) * Cfg::LDA_S + j * 8;
                        fb[j] = Cfg::kComplex ? Ad[2 * e + PASS] : Ad[e];
                    }
#pragma unroll
                    for (int i = 0; i < Cfg::NF; ++i)
#pragma unroll
                        for (int j = 0; j < Cfg::MF; ++j) {
                            if constexpr (Cfg::kComplex) {
                                // (A*B)^T = B^T A^T. Pass 0: Ar*Br -> acc0, Ar*Bi -> acc1.
                                // Pass 1: Ai*Bi -> acc0, Ai*Br -> acc1.
                                if constexpr (PASS == 0) {
                                    dmma_16x8x4(acc0[i][j], fa0[i].x, fa1[i].x, fb[j]);
                                    dmma_16x8x4(acc1[i][j], fa0[i].y, fa1[i].y, fb[j]);
                                } else {
                                    dmma_16x8x4(acc0[i][j], fa0[i].y, fa1[i].y, fb[j]);
                                    dmma_16x8x4(acc1[i][j], fa0[i].x, fa1[i].x, fb[j]);
                                }
                            } else {
                                dmma_16x8x4(acc0[i][j], fa0[i], fa1[i], fb[j]);
                            }
                        }
                }
            };
            if (pass == 0) mma_step(std::integral_constant<int, 0>{});
            else mma_step(std::integral_constant<int, 1>{});
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);

            if constexpr (SPLIT) {
                // The unit's slab ends here: its raw product goes to the
                // unit's plane (complex: P and Q of this pass side by side).
                if (q + 1 < u.iters) continue;
                const size_t at0 = (size_t)u.part * P.M * P.N;
#pragma unroll
                for (int i = 0; i < Cfg::NF; ++i)
#pragma unroll
                    for (int j = 0; j < Cfg::MF; ++j) {
                        const int m = m0 + wm * Cfg::WM + j * 8 + 2 * t;
                        if (m >= P.M) continue;
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int n = n0 + wn * Cfg::WN + i * 16 + g + 8 * h;
                            if (n >= P.N) continue;
                            const size_t at = at0 + (size_t)n * P.M + m;
                            if constexpr (Cfg::kComplex) {
                                double2* dst = reinterpret_cast<double2*>(P.S) + at;
                                dst[0] = make_double2(acc0[i][j][2 * h], acc1[i][j][2 * h]);
                                dst[1] = make_double2(acc0[i][j][2 * h + 1], acc1[i][j][2 * h + 1]);
                            } else {
                                *reinterpret_cast<double2*>(reinterpret_cast<double*>(P.S) + at) =
                                    make_double2(acc0[i][j][2 * h], acc0[i][j][2 * h + 1]);
                            }
                        }
                    }
                zero_acc();
                continue;
            }

            const bool slab_end = ((kt + 1) % slab == 0) || (kt + 1 == nk);
            if (!slab_end) continue;
            const bool first = (kt + 1) <= slab;  // first slab of this pass
            const bool last = (kt + 1 == nk) && (pass == PASSES - 1);

            // Fold the slab into C (real) or into P + iQ (complex). Real: for
            // each fragment row i, the C values are loaded first and the folds
            // and stores follow, so the loads overlap one another (measured
            // faster). Complex: each value is loaded where it is folded; a
            // gather there measured slower, the accumulators already holding
            // 128 registers.
#pragma unroll
            for (int i = 0; i < Cfg::NF; ++i) {
                double2 cur[Cfg::kComplex ? 1 : Cfg::MF][2];
                if constexpr (!Cfg::kComplex) {
                    const bool load_c = !first || br != 0.0;
#pragma unroll
                    for (int j = 0; j < Cfg::MF; ++j)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int m = m0 + wm * Cfg::WM + j * 8 + 2 * t;
                            const int n = n0 + wn * Cfg::WN + i * 16 + g + 8 * h;
                            cur[j][h] = make_double2(0.0, 0.0);
                            if (m < P.M && n < P.N && load_c)
                                cur[j][h] = *reinterpret_cast<const double2*>(reinterpret_cast<const double*>(P.C) +
                                                                               (size_t)n * P.ldc + m);
                        }
                }
#pragma unroll
                for (int j = 0; j < Cfg::MF; ++j) {
                    int m = m0 + wm * Cfg::WM + j * 8 + 2 * t;
                    if (m >= P.M) continue;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        int n = n0 + wn * Cfg::WN + i * 16 + g + 8 * h;
                        if (n >= P.N) continue;
                        if constexpr (!Cfg::kComplex) {
                            double* dst = reinterpret_cast<double*>(P.C) + (size_t)n * P.ldc + m;
                            double2 cur0 = cur[j][h];
                            // ScaleC (Gemm.cs:187-203): beta == 0 overwrites (cur0 is zero then).
                            if (first && br != 0.0 && br != 1.0)
                                cur0 = make_double2(mul_rn(cur0.x, br), mul_rn(cur0.y, br));
                            double2 out;
                            out.x = fma(ar, acc0[i][j][2 * h], cur0.x);
                            out.y = fma(ar, acc0[i][j][2 * h + 1], cur0.y);
                            *reinterpret_cast<double2*>(dst) = out;
                        } else {
                            double2* W = reinterpret_cast<double2*>(P.W ? P.W : P.C) + (size_t)n * (P.W ? P.ldw : P.ldc) + m;
                            double2* C = reinterpret_cast<double2*>(P.C) + (size_t)n * P.ldc + m;
#pragma unroll
                            for (int e = 0; e < 2; ++e) {
                                double pacc = acc0[i][j][2 * h + e];
                                double qacc = acc1[i][j][2 * h + e];
                                double2 pq;
                                if (pass == 0) {
                                    // real = Ar*Br (alpha 1, beta 0), imag = Ar*Bi (alpha 1, beta 0)
                                    double2 prev = first ? make_double2(0.0, 0.0) : W[e];
                                    pq = make_double2(fma(1.0, pacc, prev.x), fma(1.0, qacc, prev.y));
                                } else {
                                    // real += -1 * Ai*Bi, imag += 1 * Ai*Br (beta 1)
                                    double2 prev = W[e];
                                    pq = make_double2(fma(-1.0, pacc, prev.x), fma(1.0, qacc, prev.y));
                                }
                                if (!last) {
                                    W[e] = pq;
                                    continue;
                                }
                                // Combine (ComplexKernels.cs:213-240): combine_4m written
                                // out, which in this kernel compiles without the spills
                                // the call form measured under ptxas.
                                const bool unit_alpha = (ar == 1.0 && ai == 0.0);
                                const bool real_alpha = (ai == 0.0);
                                const bool zero_beta = (br == 0.0 && bi == 0.0);
                                const bool unit_beta = (br == 1.0 && bi == 0.0);
                                double pr, pi;
                                if (unit_alpha) {
                                    pr = pq.x;
                                    pi = pq.y;
                                } else if (real_alpha) {
                                    pr = mul_rn(ar, pq.x);
                                    pi = mul_rn(ar, pq.y);
                                } else {
                                    pr = sub_rn(mul_rn(ar, pq.x), mul_rn(ai, pq.y));
                                    pi = add_rn(mul_rn(ai, pq.x), mul_rn(ar, pq.y));
                                }
                                double2 o;
                                if (zero_beta) {
                                    o = make_double2(pr, pi);
                                } else {
                                    double2 c = C[e];
                                    if (unit_beta) {
                                        o = make_double2(add_rn(c.x, pr), add_rn(c.y, pi));
                                    } else {
                                        double cr = sub_rn(mul_rn(br, c.x), mul_rn(bi, c.y));
                                        double ci = add_rn(mul_rn(bi, c.x), mul_rn(br, c.y));
                                        o = make_double2(add_rn(cr, pr), add_rn(ci, pi));
                                    }
                                }
                                C[e] = o;
                            }
                        }
                    }
                }
            }
            zero_acc();
        }
    }
}

// Folds a slab-split product's planes into C in slab order, with the same
// operations the unsplit kernel applies at each slab end, so C gets the same
// bits. Real: C scaled by beta (ScaleC, Gemm.cs:187-203), then
// c = fma(alpha, slab, c) slab by slab. Complex: P and Q summed over pass 0's
// slabs from zero, pass 1's folded in (P -= Ai*Bi, Q += Ai*Br), then Combine.
// One thread per element, consecutive threads on consecutive rows.
template <bool CPLX>
__global__ void __launch_bounds__(256) slab_fold_kernel(const __grid_constant__ GemmProblem p) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = blockIdx.y;
    if (m >= p.M) return;
    const size_t plane = (size_t)p.M * p.N;
    const size_t at = (size_t)n * p.M + m;
    if constexpr (!CPLX) {
        double* c = reinterpret_cast<double*>(p.C) + (size_t)n * p.ldc + m;
        double x = 0.0;  // beta == 0 overwrites
        if (p.beta_re != 0.0) {
            x = *c;
            if (p.beta_re != 1.0) x = mul_rn(x, p.beta_re);
        }
        const double* s = reinterpret_cast<const double*>(p.S) + at;
        for (int k = 0; k < p.slabs; ++k) x = fma(p.alpha_re, s[k * plane], x);
        *c = x;
    } else {
        const double2* s = reinterpret_cast<const double2*>(p.S) + at;
        double2 pq = make_double2(0.0, 0.0);
        for (int k = 0; k < p.slabs; ++k) {
            const double2 v = s[k * plane];
            pq = make_double2(fma(1.0, v.x, pq.x), fma(1.0, v.y, pq.y));
        }
        for (int k = p.slabs; k < 2 * p.slabs; ++k) {
            const double2 v = s[k * plane];
            pq = make_double2(fma(-1.0, v.x, pq.x), fma(1.0, v.y, pq.y));
        }
        double2* c = reinterpret_cast<double2*>(p.C) + (size_t)n * p.ldc + m;
        *c = combine_4m(pq, p.alpha_re, p.alpha_im, p.beta_re, p.beta_im, c);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

namespace {

using RealBig = GemmCfg<false, 4, 2, 4>;    // 128 x 128 tiles, 8 math warps
using RealSmall = GemmCfg<false, 2, 1, 4>;  // 64 x 64 tiles, 2 math warps
using CplxBig = GemmCfg<true, 4, 2, 3>;     // 128 x 64 tiles, 8 math warps
using CplxSmall = GemmCfg<true, 2, 2, 4>;   // 64 x 64 tiles, 4 math warps

// The math warpgroups' register increase can only be met when the kernel is
// launched with exactly the allocation the split assumes; with any other
// allocation they would wait forever, so such a build is refused.
template <class Cfg, bool SPLIT>
void check_register_split() {
    if constexpr (Cfg::kSplitRegs) {
        cudaFuncAttributes fa{};
        TNS_CUDA(cudaFuncGetAttributes(&fa, gemm_dmma_kernel<Cfg, SPLIT>));
        if (fa.numRegs != Cfg::kLaunchRegs)
            fail(TNS_E_DEVICE, "GEMM kernel built with " + std::to_string(fa.numRegs) +
                                   " registers per thread; its register split needs " +
                                   std::to_string(Cfg::kLaunchRegs));
    }
}

// A 2-D double-precision TMA descriptor: `rows` x `cols` doubles, column
// stride `ld_bytes`, boxes of box_rows x box_cols, zero fill outside.
void encode_map(CUtensorMap* map, const void* base, uint64_t rows, uint64_t cols, uint64_t ld_bytes,
                uint32_t box_rows, uint32_t box_cols) {
    cuuint64_t dims[2] = {rows, cols};
    cuuint64_t strides[1] = {ld_bytes};
    cuuint32_t box[2] = {box_rows, box_cols};
    cuuint32_t elem[2] = {1, 1};
    // The driver's encoder, looked up through the runtime so that the library
    // loads (and its host-only entry points work) where no driver is present.
    static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) fail(TNS_E_DEVICE, "the CUDA driver does not provide cuTensorMapEncodeTiled");
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(base), dims, strides, box, elem,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(TNS_E_DEVICE, "TMA descriptor encoding failed (CUresult " + std::to_string((int)r) + ")");
}

// Descriptors of one problem's operands for configuration Cfg.
template <class Cfg>
GemmMaps encode_maps(const GemmProblem& p) {
    GemmMaps m;
    encode_map(&m.a, p.A, (uint64_t)Cfg::DPE * p.M, (uint64_t)p.K, (uint64_t)p.lda * Cfg::ESZ,
               Cfg::DPE * Cfg::LDA_S, Cfg::BK);
    encode_map(&m.b, p.B, (uint64_t)Cfg::DPE * p.K, (uint64_t)p.N, (uint64_t)p.ldb * Cfg::ESZ,
               Cfg::DPE * Cfg::LDB_S, Cfg::BN);
    return m;
}

// One launch of configuration Cfg over `probs`. SPLIT: every problem carries
// its slab planes (S, slabs) and `tail` enqueues the fold that follows the
// kernel, inside the launch's timing events.
template <class Cfg, bool SPLIT = false>
void launch_cfg(Context& ctx, std::vector<GemmProblem>& probs, const std::function<void()>& tail = {}) {
    static std::atomic<bool> configured[64];
    int dev = ctx.device;
    if (!configured[dev].load(std::memory_order_acquire)) {
        TNS_CUDA(cudaFuncSetAttribute(gemm_dmma_kernel<Cfg, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      Cfg::SMEM));
        check_register_split<Cfg, SPLIT>();
        configured[dev].store(true, std::memory_order_release);
    }
    int total = 0;
    for (auto& p : probs) {
        p.tiles_m = (p.M + Cfg::BM - 1) / Cfg::BM;
        p.tiles_n = (p.N + Cfg::BN - 1) / Cfg::BN;
        p.tile_begin = total;
        total += p.tiles_m * p.tiles_n * (SPLIT ? p.slabs * (Cfg::kComplex ? 2 : 1) : 1);
    }
    if (total == 0) return;
    GemmLaunch L{};
    L.nprob = (int)probs.size();
    L.total_tiles = total;
    L.err = ctx.d_err;
    L.tiles = ctx.d_tiles;
    TNS_CUDA(cudaMemsetAsync(ctx.d_tiles, 0, sizeof(unsigned long long), ctx.stream));
    if (probs.size() <= 4) {
        for (size_t i = 0; i < probs.size(); ++i) {
            L.inl[i] = probs[i];
            L.inl_maps[i] = encode_maps<Cfg>(probs[i]);
        }
        L.list = nullptr;
        L.maps_list = nullptr;
    } else {
        std::vector<GemmMaps> maps(probs.size());
        for (size_t i = 0; i < probs.size(); ++i) maps[i] = encode_maps<Cfg>(probs[i]);
        L.list = static_cast<const GemmProblem*>(ctx.upload(probs.data(), sizeof(GemmProblem) * probs.size()));
        L.maps_list = static_cast<const GemmMaps*>(ctx.upload(maps.data(), sizeof(GemmMaps) * maps.size()));
    }
    int ctas_per_sm = 1;
    TNS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas_per_sm, gemm_dmma_kernel<Cfg, SPLIT>, Cfg::THREADS,
                                                           Cfg::SMEM));
    int grid = std::min(total, std::max(1, ctas_per_sm) * ctx.num_sms);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ctx.timing) {
        e0 = ctx.take_event();
        e1 = ctx.take_event();
        TNS_CUDA(cudaEventRecord(e0, ctx.stream));
    }
    gemm_dmma_kernel<Cfg, SPLIT><<<grid, Cfg::THREADS, Cfg::SMEM, ctx.stream>>>(L);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
    ctx.gemm_launches++;
    if (tail) tail();
    for (auto& p : probs) {
        ctx.gemm_flops += (Cfg::kComplex ? 8.0 : 2.0) * (double)(p.work > 0 ? p.work : (long long)p.M * p.N * p.K);
        const bool reads_c = p.beta_re != 0.0 || p.beta_im != 0.0;
        ctx.gemm_bytes += (Cfg::kComplex ? 16.0 : 8.0) *
                          ((double)p.M * p.K + (double)p.K * p.N + (double)p.M * p.N * (reads_c ? 2.0 : 1.0));
    }
    if (ctx.timing) {
        TNS_CUDA(cudaEventRecord(e1, ctx.stream));
        ctx.gemm_events.emplace_back(e0, e1);
        if (ctx.gemm_events.size() > 4096) ctx.drain_events();
    }
}

void check_problem(const GemmProblem& p, bool cplx) {
    int esz = cplx ? 16 : 8;
    auto aligned = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    bool ok = p.M >= 0 && p.N >= 0 && p.K >= 0 && (p.M % 2 == 0) && (p.N % 2 == 0) && (p.K % 16 == 0) &&
              p.kc > 0 && (p.kc % 16 == 0) && aligned(p.A) && aligned(p.B) && aligned(p.C) &&
              ((size_t)p.lda * esz) % 16 == 0 && ((size_t)p.ldb * esz) % 16 == 0 && ((size_t)p.ldc * esz) % 16 == 0 &&
              p.lda >= p.M && p.ldb >= p.K && p.ldc >= p.M && (!p.W || (aligned(p.W) && p.ldw >= p.M));
    if (!ok) fail(TNS_E_ARGUMENT, "internal GEMM operand violates the bulk-copy layout contract");
}

}  // namespace

namespace {

// Slab planes of a slab-split product stay below this size.
constexpr size_t kSlabPlaneBytes = size_t(512) << 20;

// One product whose tiles leave SMs idle and whose K spans several KC slabs:
// each tile's slabs (and passes) run as separate units, so more CTAs work at
// once, each unit's raw slab product goes to its own plane, and a fold kernel
// adds the slabs into C in slab order with the operations the unsplit kernel
// applies at each slab end (the same bits). False when the split does not
// apply.
template <class Big, class Small>
bool slab_split_launch(Context& ctx, const GemmProblem& p0, long long tiles_big) {
    constexpr bool CPLX = Big::kComplex;
    constexpr int passes = CPLX ? 2 : 1;
    const int slabs = (p0.K + p0.kc - 1) / p0.kc;
    const size_t bytes = (size_t)passes * slabs * p0.M * p0.N * Big::ESZ;
    if (slabs < 2 || tiles_big >= ctx.num_sms || bytes > kSlabPlaneBytes) return false;
    DBuf planes(ctx, bytes);
    GemmProblem p = p0;
    p.S = planes.p;
    p.slabs = slabs;
    p.W = nullptr;
    p.ldw = 0;
    std::vector<GemmProblem> v{p};
    auto fold = [&] {
        slab_fold_kernel<CPLX><<<dim3((p.M + 255) / 256, p.N), 256, 0, ctx.stream>>>(p);
        TNS_CUDA(cudaGetLastError());
        ctx.kernel_launches++;
    };
    if (tiles_big * slabs * passes >= ctx.num_sms) launch_cfg<Big, true>(ctx, v, fold);
    else launch_cfg<Small, true>(ctx, v, fold);
    return true;
}

void gemm_run(Context& ctx, std::vector<GemmProblem>& probs, bool cplx, bool slab_split) {
    std::vector<GemmProblem> work;
    work.reserve(probs.size());
    for (auto& p0 : probs) {
        GemmProblem p = p0;
        if (p.kc <= 0) p.kc = reference_kc(p.work > 0 ? p.work : (long long)p.M * p.N * p.K);
        check_problem(p, cplx);
        if (p.M == 0 || p.N == 0) continue;
        if (p.K == 0) {
            // No product: C := beta*C.
            scale_inplace(ctx, p.C, p.M, p.N, p.ldc, cplx, p.beta_re, p.beta_im);
            continue;
        }
        work.push_back(p);
    }
    if (work.empty()) return;
    // Heaviest tiles (deepest K) first: CTAs take tiles in list order as they
    // free up, so the launch ends on light tiles.
    std::stable_sort(work.begin(), work.end(), [](const GemmProblem& x, const GemmProblem& y) { return x.K > y.K; });
    // Big tiles only when they fill the machine, or as the autotuner found.
    long long tiles = 0;
    int depth = 0;
    bool overwrite = true;  // every C is overwritten (beta = 0): a trial may run twice
    for (auto& p : work) {
        tiles += cplx ? (long long)((p.M + CplxBig::BM - 1) / CplxBig::BM) * ((p.N + CplxBig::BN - 1) / CplxBig::BN)
                      : (long long)((p.M + RealBig::BM - 1) / RealBig::BM) * ((p.N + RealBig::BN - 1) / RealBig::BN);
        depth = std::max(depth, p.K);
        if (p.beta_re != 0.0 || p.beta_im != 0.0) overwrite = false;
    }
    if (slab_split && work.size() == 1 &&
        (cplx ? slab_split_launch<CplxBig, CplxSmall>(ctx, work[0], tiles)
              : slab_split_launch<RealBig, RealSmall>(ctx, work[0], tiles)))
        return;
    std::vector<DBuf> scratch;
    scratch.reserve(work.size());
    for (auto& p : work) {
        if (cplx && !p.W && !(p.alpha_re == 1.0 && p.alpha_im == 0.0 && p.beta_re == 0.0 && p.beta_im == 0.0)) {
            // P + iQ need their own storage when the combine is not a plain copy.
            scratch.emplace_back(ctx, (size_t)p.M * p.N * 16);
            p.W = scratch.back().p;
            p.ldw = p.M;
        }
    }
    auto run = [&](int big) {
        if (cplx) big ? launch_cfg<CplxBig>(ctx, work) : launch_cfg<CplxSmall>(ctx, work);
        else big ? launch_cfg<RealBig>(ctx, work) : launch_cfg<RealSmall>(ctx, work);
    };
    int variant = tiles >= ctx.num_sms ? 1 : 0;
    if (ctx.autotune) {
        const TuneKind kind = cplx ? TuneKind::kDmmaComplex : TuneKind::kDmmaReal;
        const int known = tuned_variant(ctx.device, kind, tiles, depth);
        if (known >= 0) {
            variant = known;
        } else if (overwrite) {
            const float small = time_launches(ctx, [&] { run(0); });
            const float big = time_launches(ctx, [&] { run(1); });  // the same values again
            record_variant(ctx.device, kind, tiles, depth, big <= small ? 1 : 0);
            ctx.autotune_trials++;
            return;
        }
    }
    run(variant);
}

}  // namespace

void gemm_grouped(Context& ctx, std::vector<GemmProblem>& probs, bool cplx) { gemm_run(ctx, probs, cplx, false); }

// One product through the public entry points: slab-split when its tiles
// alone would leave SMs idle.
void gemm(Context& ctx, const GemmProblem& p, bool cplx) {
    std::vector<GemmProblem> v{p};
    gemm_run(ctx, v, cplx, true);
}

namespace {
template <class Cfg>
void launch_detached(cudaStream_t stream, int num_sms, int* d_err, GemmProblem p) {
    TNS_CUDA(cudaFuncSetAttribute(gemm_dmma_kernel<Cfg, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
    check_register_split<Cfg, false>();
    p.tiles_m = (p.M + Cfg::BM - 1) / Cfg::BM;
    p.tiles_n = (p.N + Cfg::BN - 1) / Cfg::BN;
    p.tile_begin = 0;
    int total = p.tiles_m * p.tiles_n;
    if (total == 0) return;
    GemmLaunch L{};
    L.inl[0] = p;
    L.inl_maps[0] = encode_maps<Cfg>(p);
    L.list = nullptr;
    L.maps_list = nullptr;
    L.nprob = 1;
    L.total_tiles = total;
    L.err = d_err;
    L.tiles = nullptr;  // no counter without a context: static round robin
    int ctas_per_sm = 1;
    TNS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas_per_sm, gemm_dmma_kernel<Cfg, false>, Cfg::THREADS,
                                                           Cfg::SMEM));
    int grid = std::min(total, std::max(1, ctas_per_sm) * num_sms);
    gemm_dmma_kernel<Cfg, false><<<grid, Cfg::THREADS, Cfg::SMEM, stream>>>(L);
    TNS_CUDA(cudaGetLastError());
}
}  // namespace

// One complex product launched on a caller's stream without a context: the
// problem's operands and its P + iQ workspace (W) are the caller's, nothing is
// allocated and nothing is uploaded (the problem travels in the launch
// parameters). Same kernel, tiles and KC rule as gemm(), always unsplit (a
// slab split's planes would need storage); the bits are the same either way.
void gemm_detached_complex(cudaStream_t stream, int device, int* d_err, const GemmProblem& p0) {
    GemmProblem p = p0;
    if (p.kc <= 0) p.kc = reference_kc(p.work > 0 ? p.work : (long long)p.M * p.N * p.K);
    check_problem(p, true);
    if (p.M == 0 || p.N == 0 || p.K == 0) return;
    int num_sms = 148;
    TNS_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    long long tiles = (long long)((p.M + CplxBig::BM - 1) / CplxBig::BM) * ((p.N + CplxBig::BN - 1) / CplxBig::BN);
    if (tiles >= num_sms) launch_detached<CplxBig>(stream, num_sms, d_err, p);
    else launch_detached<CplxSmall>(stream, num_sms, d_err, p);
}

}  // namespace tns
