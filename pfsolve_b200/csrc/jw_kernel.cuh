// jw_kernel.cuh -- the fused Jones-Worland step for sm_100a.
//
// One JW step per right-hand side (PfSolve_shaderGen_JonesWorlandMV,
// PfSolve/pfSolve_CodeGen/pfSolve_KernelsLevel2/pfSolve_JonesWorland.h:38-408):
//
//     x = diag(s) * M^{-1} * (V * A * b),   x[0] *= scaleC when a solve runs
//
//   A : optional general band matrix of a fused dgbmv app (band-major storage,
//       pfSolve_KernelsLevel1/pfSolve_MatVecMul.h:383-446),
//   V : the JW matvec (identity, diagonal, upper or lower bidiagonal;
//       pfSolve_MatVecMul.h:28-133),
//   M : unit-diagonal lower/upper bidiagonal or tridiagonal solve
//       (pfSolve_KernelsLevel1/pfSolve_TridiagonalSolve.h:1578-1929),
//   s : optional per-row Scale factor of a fused block app
//       (pfSolve_KernelsLevel1/pfSolve_RegistersScaleC.h:27-201).
//
// Design (B200-first, not the reference's codegen):
//  * All systems of a launch share one matrix, so each thread group factors it
//    once (prologue) and keeps per-row coefficients in registers for every
//    system it processes.  The product V*A is folded into one band of
//    KL+KU+1 weights per row, the tridiagonal LU is computed once, and the
//    per-system work is ~5 FMAs per row plus two affine scans.
//  * A group of W warps owns one system at a time; thread t owns rows
//    [R*t, R*t+R) (partition method).  The within-chunk recurrences run in
//    registers; the chunk-boundary couplings are resolved by Kogge-Stone scans
//    of affine maps over warp shuffles, then over warps through shared memory.
//  * The tridiagonal LU pivots d'_i = 1 - a_i c_{i-1} / d'_{i-1} form a
//    Moebius recurrence; the prologue evaluates it in parallel as a scan of
//    exactly renormalised 2x2 matrix products.
//  * Right-hand sides stream global -> shared with cp.async (zero-fill gives
//    the zeropad keep-window and out-of-range rows for free), double-buffered
//    per warp, into an XOR-swizzled layout that is conflict-free for both the
//    coalesced write and the blocked (per-thread chunk) read.
//  * PREC_MIXED: FP64 storage, the solve factors rounded to FP32 and applied
//    in FP32; the residual r = V*A*b - M*x and the correction accumulation run
//    in FP64 (iterative refinement, all on chip: b is never re-read).
//  * PREC_F32 / PREC_F64_F32MEM: FP32 storage (right-hand sides and bands),
//    FP32 or FP64 arithmetic (the reference's precision 0 and its
//    doublePrecisionFloatMemory).  The coefficients are still formed in FP64
//    from the FP32 bands, then held in the arithmetic type.
#pragma once
#include <type_traits>

#include "common.cuh"
#include "jw_types.h"

namespace pfb {

template <int R, int KL, int KU, int SV, int LIN, int LOUT, bool SCALE, int PREC = PREC_F64, bool TBL = false>
struct JwCfg {
    static constexpr int kR = R, kKL = KL, kKU = KU, kSV = SV, kLIN = LIN, kLOUT = LOUT, kPrec = PREC;
    static constexpr bool kScale = SCALE;
    static constexpr bool kCplx = (LIN != LAY_REAL);
    static constexpr bool kF32Mem = prec_f32_storage(PREC);  // FP32 storage
    static constexpr bool kF32 = (PREC == PREC_F32);          // FP32 arithmetic
    using MS = typename std::conditional<kF32, float, double>::type;  // arithmetic scalar
    using T = typename std::conditional<kF32Mem, float, double>::type;  // storage scalar
    using V = typename std::conditional<kCplx, typename Vec2Of<MS>::type, MS>::type;
    using TS = typename std::conditional<kCplx, typename Vec2Of<T>::type, T>::type;  // staged element
    using VF = typename Lower<V>::type;
    static constexpr int NB = KL + KU + 1;
    static constexpr int SEG = 32 * R + KL + KU;  // elements per warp buffer
    static constexpr bool kFwd = (SV == SV_LOWER || SV == SV_TRI);
    static constexpr bool kBwd = (SV == SV_UPPER || SV == SV_TRI);
    static constexpr bool kMixed = (PREC == PREC_MIXED) && (SV != SV_NONE);
    static constexpr int NF = kFwd ? R : 1;
    static constexpr int NBW = kBwd ? R : 1;
    // Coefficients in a CTA-shared table: planes w[0..NB), l, h, sc, each
    // [R][T] doubles (T threads per group) -- lane-contiguous, conflict-free.
    static constexpr bool kTbl = TBL && !kMixed && PREC == PREC_F64;
    static constexpr int P_L = NB, P_H = NB + (kFwd ? 1 : 0), P_SC = P_H + (kBwd ? 1 : 0);
    static constexpr int NPLANES = P_SC + (SCALE ? 1 : 0);
    // Register-resident coefficients need up to 255 registers: 256-thread
    // CTAs.  Table variants keep data only: up to 512 threads (<= 128 regs).
    static constexpr int kMaxThreads = kTbl ? 512 : 256;
};

constexpr int kScratchPerWarp = 32;  // doubles

// Shared memory per warp: two segment buffers (16-byte aligned).  The scratch
// (kScratchPerWarp doubles per warp) follows all warp buffers.
template <class C>
__host__ __device__ constexpr size_t jw_smem_per_warp()
{
    return ((2 * (size_t)C::SEG * sizeof(typename C::TS)) + 15) / 16 * 16;
}

template <class C>
__host__ __device__ constexpr size_t jw_table_bytes(int W)
{
    return C::kTbl ? (size_t)C::NPLANES * C::kR * 32 * W * sizeof(double) : 0;
}

template <class C>
__host__ size_t jw_smem_bytes(int W, int G)
{
    return jw_table_bytes<C>(W) + (size_t)G * W * jw_smem_per_warp<C>() +
           (size_t)G * W * kScratchPerWarp * sizeof(double);
}

// Storage position of row i in the reference's band order (reorder_i0,
// pfSolve_Plan_JonesWorland.h:66-142): register-major within each piece of
// perm_piece rows (the whole system when perm_piece == 0).
__device__ __forceinline__ int64_t band_pos(const JwOperator& op, int64_t i)
{
    if (op.alt) return (i % op.alt_R) * op.alt_T + op.alt_h * (op.alt_T >> 1) + i / op.alt_R;
    if (!op.perm) return i;
    int64_t base = 0, li = i, m = op.perm_m, ce = op.perm_ceil, fl = op.perm_floor;
    if (op.perm_piece) {
        const int64_t piece = i / op.perm_piece;
        base = piece * op.perm_piece;
        li = i - base;
        if (base + op.perm_piece > op.M) {
            m = op.perm_lm;
            ce = op.perm_lceil;
            fl = op.perm_lfloor;
        }
    }
    const int64_t t = li / op.perm_r, j = li - t * op.perm_r;
    return base + t + ((j < m) ? j * ce : m * ce + (j - m) * fl);
}

// Band entry at element index idx: FP64, or FP32 widened (bands32).
__device__ __forceinline__ double band_at(const JwOperator& op, const double* base, int64_t idx)
{
    return op.bands32 ? (double)__ldg(reinterpret_cast<const float*>(base) + idx) : __ldg(base + idx);
}

__device__ __forceinline__ double band(const JwOperator& op, int64_t off, int64_t i)
{
    return band_at(op, op.bands, off + band_pos(op, i));
}

// Per-row Scale factor, runtime-scaleC form (pfSolve_RegistersScaleC.h:27-201).
__device__ __forceinline__ double scale_factor(int kind, int64_t x, int L, double s)
{
    double X = (double)x;
    switch (kind) {
    case 1: return s;
    case 2: return 2.0 * (X + L + 1.0) * sqrt((X + 1.0) / (X + s + L + 1.5));
    case 3:
        return 4.0 * (X + L + 2.0) * (X + L + 3.0) *
               sqrt((X + 1.0) * (X + 2.0) / ((X + s + L + 2.5) * (X + s + L + 3.5)));
    case 4: return (4.0 * L + 6.0) * (X + L + 1.0) * sqrt((X + 1.0) / (X + s + L + 1.5));
    default: return 1.0;
    }
}

// Per-thread coefficients of one matrix, in registers or in the CTA-shared
// table.  FP64 path: the solve scaling is folded into w.  Mixed path: w stays
// unscaled (it forms g = V*A*b), the solve factors live in FP32 and the
// unit-diagonal solve bands in FP64 for the residual.  The in-chunk products of
// the recurrences (-l and -h) are formed on the fly by the solve.
template <class C>
struct JwCoef {
    using S = typename std::conditional<C::kMixed || C::kF32, float, double>::type;
    using WT = typename C::MS;  // matvec weights and Scale factors: the arithmetic type
    static constexpr int RR = C::kTbl ? 1 : C::kR;
    WT w_[C::NB][RR];
    S m_[C::kMixed ? C::kR : 1];
    S l_[C::kTbl ? 1 : C::NF];
    S h_[C::kTbl ? 1 : C::NBW];
    double al_[C::kMixed ? C::NF : 1];   // M's sub-diagonal (residual)
    double cu_[C::kMixed ? C::NBW : 1];  // M's super-diagonal (residual)
    WT sc_[(C::kScale && !C::kTbl) ? C::kR : 1];
    const double* tbl;  // table mode: plane p, row j of thread tt at tbl[(p*R + j)*T + tt]
    int T, tt;

    __device__ __forceinline__ double t_(int p, int j) const { return tbl[(p * C::kR + j) * T + tt]; }
    __device__ __forceinline__ WT w(int k, int j) const
    {
        if constexpr (C::kTbl) return t_(k, j);
        else return w_[k][j];
    }
    __device__ __forceinline__ S l(int j) const
    {
        if constexpr (C::kTbl) return t_(C::P_L, j);
        else return l_[j];
    }
    __device__ __forceinline__ S h(int j) const
    {
        if constexpr (C::kTbl) return t_(C::P_H, j);
        else return h_[j];
    }
    __device__ __forceinline__ WT sc(int j) const
    {
        if constexpr (C::kTbl) return t_(C::P_SC, j);
        else return sc_[j];
    }
};

// Cross-warp scratch: kScratchPerWarp doubles per warp,
//   [0, 8)   forward scan aggregates  (2 slots x {A, -, B.x, B.y})
//   [8, 16)  backward scan aggregates
//   [16, 24) neighbour exchange       (2 slots x {first.x, first.y, last.x, last.y})
//   [24, 28) factorisation scan (2x2 matrix)
// Every cross-warp operation bumps `seq` and uses slot seq & 1: a warp can only
// rewrite a slot after passing the barrier of the next operation, which every
// other warp reaches after reading the slot.
struct GroupCtx {
    int lane, wg, W, nthr, bar_id, seq;
    double* scratch;  // scratch of warp 0 of this group; warp w at scratch + kScratchPerWarp*w
    __device__ __forceinline__ double* warp_area(int w) const { return scratch + kScratchPerWarp * w; }
};

template <class V>
__device__ __forceinline__ void store_v(double* p, V v) { *reinterpret_cast<V*>(p) = v; }
template <class V>
__device__ __forceinline__ V load_v(const double* p) { return *reinterpret_cast<const V*>(p); }

// Exclusive scan of affine maps y = B + A*x over the group, in row order
// (forward) or reverse row order (backward).  Returns the value entering this
// thread's chunk; the value entering the whole system is zero.
template <class V, class S, bool FORWARD>
__device__ __forceinline__ V group_affine_scan(GroupCtx& g, S A, V B)
{
    using O = VOps<V>;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        S Ap = FORWARD ? shfl_up_s<S>(A, d) : shfl_down_s<S>(A, d);
        V Bp = FORWARD ? O::shfl_up(B, d) : O::shfl_down(B, d);
        bool take = FORWARD ? (g.lane >= d) : (g.lane + d < 32);
        if (take) {
            B = O::fma(A, Bp, B);
            A = A * Ap;
        }
    }
    S Ae = FORWARD ? shfl_up_s<S>(A, 1) : shfl_down_s<S>(A, 1);
    V Be = FORWARD ? O::shfl_up(B, 1) : O::shfl_down(B, 1);
    const bool first = FORWARD ? (g.lane == 0) : (g.lane == 31);
    if (first) {
        Ae = S(1);
        Be = O::zero();
    }
    V win = O::zero();
    if (g.W > 1) {
        const int slot = (FORWARD ? 0 : 8) + 4 * (g.seq & 1);
        const bool agg = FORWARD ? (g.lane == 31) : (g.lane == 0);
        if (agg) {
            double* my = g.warp_area(g.wg) + slot;
            store_v<S>(my, A);
            store_v<V>(my + 2, B);
        }
        __syncwarp();
        group_bar(g.bar_id, g.nthr);
        if (FORWARD) {
            for (int w = 0; w < g.wg; ++w) {
                const double* o = g.warp_area(w) + slot;
                win = O::fma(load_v<S>(o), win, load_v<V>(o + 2));
            }
        } else {
            for (int w = g.W - 1; w > g.wg; --w) {
                const double* o = g.warp_area(w) + slot;
                win = O::fma(load_v<S>(o), win, load_v<V>(o + 2));
            }
        }
        g.seq++;
    }
    return O::fma(Ae, win, Be);
}

// The multipliers of an affine scan whose per-thread multipliers A are the
// same for every system (products of a coefficient table that all systems
// share): each lane's multiplier at each shuffle level, the multiplier of its
// exclusive result and its warp's aggregate, formed once so that a system's
// scan (group_affine_scan_pre) shuffles only its values.
template <class S>
struct ScanMul {
    S lev[5];
    S Ae;
    S Aw;
};

template <class S, bool FORWARD>
__device__ __forceinline__ ScanMul<S> scan_multipliers(const GroupCtx& g, S A)
{
    ScanMul<S> m;
    int i = 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1, ++i) {
        m.lev[i] = A;
        const S Ap = FORWARD ? shfl_up_s<S>(A, d) : shfl_down_s<S>(A, d);
        const bool take = FORWARD ? (g.lane >= d) : (g.lane + d < 32);
        if (take) A = A * Ap;
    }
    m.Aw = A;
    const S Ae = FORWARD ? shfl_up_s<S>(A, 1) : shfl_down_s<S>(A, 1);
    const bool first = FORWARD ? (g.lane == 0) : (g.lane == 31);
    m.Ae = first ? S(1) : Ae;
    return m;
}

// group_affine_scan with the multipliers formed by scan_multipliers.
template <class V, class S, bool FORWARD>
__device__ __forceinline__ V group_affine_scan_pre(GroupCtx& g, const ScanMul<S>& m, V B)
{
    using O = VOps<V>;
    int i = 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1, ++i) {
        const V Bp = FORWARD ? O::shfl_up(B, d) : O::shfl_down(B, d);
        const bool take = FORWARD ? (g.lane >= d) : (g.lane + d < 32);
        if (take) B = O::fma(m.lev[i], Bp, B);
    }
    V Be = FORWARD ? O::shfl_up(B, 1) : O::shfl_down(B, 1);
    const bool first = FORWARD ? (g.lane == 0) : (g.lane == 31);
    if (first) Be = O::zero();
    V win = O::zero();
    if (g.W > 1) {
        const int slot = (FORWARD ? 0 : 8) + 4 * (g.seq & 1);
        const bool agg = FORWARD ? (g.lane == 31) : (g.lane == 0);
        if (agg) {
            double* my = g.warp_area(g.wg) + slot;
            store_v<S>(my, m.Aw);
            store_v<V>(my + 2, B);
        }
        __syncwarp();
        group_bar(g.bar_id, g.nthr);
        if (FORWARD) {
            for (int w = 0; w < g.wg; ++w) {
                const double* o = g.warp_area(w) + slot;
                win = O::fma(load_v<S>(o), win, load_v<V>(o + 2));
            }
        } else {
            for (int w = g.W - 1; w > g.wg; --w) {
                const double* o = g.warp_area(w) + slot;
                win = O::fma(load_v<S>(o), win, load_v<V>(o + 2));
            }
        }
        g.seq++;
    }
    return O::fma(m.Ae, win, Be);
}

// Two independent affine scans at once, elementwise in .x and .y (the two
// ALT systems of a staged row set): one shuffle chain and one group barrier
// instead of two.  Same slots as group_affine_scan (a double2 multiplier and
// a double2 value fill the 4 doubles of a slot).
template <bool FORWARD>
__device__ __forceinline__ double2 group_affine_scan2(GroupCtx& g, double2 A, double2 B)
{
    using O = VOps<double2>;
    auto fma2 = [](double2 a, double2 v, double2 w) {
        return make_double2(__fma_rn(a.x, v.x, w.x), __fma_rn(a.y, v.y, w.y));
    };
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double2 Ap = FORWARD ? O::shfl_up(A, d) : O::shfl_down(A, d);
        const double2 Bp = FORWARD ? O::shfl_up(B, d) : O::shfl_down(B, d);
        const bool take = FORWARD ? (g.lane >= d) : (g.lane + d < 32);
        if (take) {
            B = fma2(A, Bp, B);
            A = make_double2(A.x * Ap.x, A.y * Ap.y);
        }
    }
    double2 Ae = FORWARD ? O::shfl_up(A, 1) : O::shfl_down(A, 1);
    double2 Be = FORWARD ? O::shfl_up(B, 1) : O::shfl_down(B, 1);
    const bool first = FORWARD ? (g.lane == 0) : (g.lane == 31);
    if (first) {
        Ae = make_double2(1.0, 1.0);
        Be = O::zero();
    }
    double2 win = O::zero();
    if (g.W > 1) {
        const int slot = (FORWARD ? 0 : 8) + 4 * (g.seq & 1);
        const bool agg = FORWARD ? (g.lane == 31) : (g.lane == 0);
        if (agg) {
            double* my = g.warp_area(g.wg) + slot;
            store_v<double2>(my, A);
            store_v<double2>(my + 2, B);
        }
        __syncwarp();
        group_bar(g.bar_id, g.nthr);
        if (FORWARD) {
            for (int w = 0; w < g.wg; ++w) {
                const double* o = g.warp_area(w) + slot;
                win = fma2(load_v<double2>(o), win, load_v<double2>(o + 2));
            }
        } else {
            for (int w = g.W - 1; w > g.wg; --w) {
                const double* o = g.warp_area(w) + slot;
                win = fma2(load_v<double2>(o), win, load_v<double2>(o + 2));
            }
        }
        g.seq++;
    }
    return fma2(Ae, win, Be);
}

// Values of the rows around this thread's chunk: x[s-1] (prev) and x[s+R]
// (next); zero outside the system.
template <class V>
__device__ __forceinline__ void group_neighbours(GroupCtx& g, V first, V last, V& prev, V& next)
{
    using O = VOps<V>;
    prev = O::shfl_up(last, 1);
    next = O::shfl_down(first, 1);
    if (g.W > 1) {
        const int slot = 16 + 4 * (g.seq & 1);
        double* my = g.warp_area(g.wg) + slot;
        if (g.lane == 0) store_v<V>(my, first);
        if (g.lane == 31) store_v<V>(my + 2, last);
        __syncwarp();
        group_bar(g.bar_id, g.nthr);
        if (g.lane == 0) prev = (g.wg > 0) ? load_v<V>(g.warp_area(g.wg - 1) + slot + 2) : O::zero();
        if (g.lane == 31) next = (g.wg < g.W - 1) ? load_v<V>(g.warp_area(g.wg + 1) + slot) : O::zero();
        g.seq++;
    } else {
        if (g.lane == 0) prev = O::zero();
        if (g.lane == 31) next = O::zero();
    }
}

// Exclusive scan of 2x2 matrix products P_t * ... * P_0 (row order) used by
// the tridiagonal factorisation.  Returns the product of all preceding chunks.
__device__ __forceinline__ void group_matrix_scan(GroupCtx& g, double& a, double& b, double& c, double& d)
{
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
        double pa = __shfl_up_sync(FULL, a, s), pb = __shfl_up_sync(FULL, b, s);
        double pc = __shfl_up_sync(FULL, c, s), pd = __shfl_up_sync(FULL, d, s);
        if (g.lane >= s) {  // mine * previous
            double na = a * pa + b * pc, nb = a * pb + b * pd;
            double nc = c * pa + d * pc, nd = c * pb + d * pd;
            a = na; b = nb; c = nc; d = nd;
            renorm2x2(a, b, c, d);
        }
    }
    double ea = __shfl_up_sync(FULL, a, 1), eb = __shfl_up_sync(FULL, b, 1);
    double ec = __shfl_up_sync(FULL, c, 1), ed = __shfl_up_sync(FULL, d, 1);
    if (g.lane == 0) { ea = 1; eb = 0; ec = 0; ed = 1; }
    double wa = 1, wb = 0, wc = 0, wd = 1;  // product of preceding warps
    if (g.W > 1) {
        double* my = g.warp_area(g.wg) + 24;
        if (g.lane == 31) { my[0] = a; my[1] = b; my[2] = c; my[3] = d; }
        __syncwarp();
        group_bar(g.bar_id, g.nthr);
        for (int w = 0; w < g.wg; ++w) {
            const double* o = g.warp_area(w) + 24;
            double na = o[0] * wa + o[1] * wc, nb = o[0] * wb + o[1] * wd;
            double nc = o[2] * wa + o[3] * wc, nd = o[2] * wb + o[3] * wd;
            wa = na; wb = nb; wc = nc; wd = nd;
            renorm2x2(wa, wb, wc, wd);
        }
        group_bar(g.bar_id, g.nthr);
    }
    a = ea * wa + eb * wc;
    b = ea * wb + eb * wd;
    c = ec * wa + ed * wc;
    d = ec * wb + ed * wd;
}

// Effective matvec weights of V*A for row i (0 <= i < M): w[q] multiplies
// row i + q - KL.  Without a fused dgbmv, V alone.
template <int KL, int NB>
__device__ __forceinline__ void jw_row_weights(const JwOperator& op, int64_t i, double (&w)[NB])
{
    const int64_t M = op.M;
#pragma unroll
    for (int k = 0; k < NB; ++k) w[k] = 0.0;
    double vl = 0, vd = 1, vu = 0;
    if (op.mvj != MVJ_NONE) vd = band(op, op.off_md, i);
    if (op.mvj == MVJ_UPPER && i + 1 < M) vu = band(op, op.off_mo, i);
    if (op.mvj == MVJ_LOWER && i >= 1) vl = band(op, op.off_mo, i);
    if (op.dgbmv == nullptr) {
        if constexpr (KL >= 1) w[KL - 1] = vl;
        w[KL] = vd;
        if constexpr (NB - KL - 1 >= 1) w[KL + 1] = vu;
    } else {
        const int kla = op.dg_lda - 1 - op.dg_ku;
        for (int pv = -1; pv <= 1; ++pv) {
            const double vp = (pv < 0) ? vl : (pv == 0 ? vd : vu);
            const int64_t p = i + pv;
            if (vp == 0.0 || p < 0 || p >= M) continue;
            for (int kk = -kla; kk <= op.dg_ku; ++kk) {
                const int64_t c = p + kk;
                if (c < 0 || c >= M || ((op.dg_skip >> (op.dg_ku - kk)) & 1)) continue;
                const double a = band_at(op, op.dgbmv, op.dg_off + (int64_t)(op.dg_ku - kk) * M + c);
                const int64_t k = c - i;  // within [-KL, KU] by construction of the plan
#pragma unroll
                for (int q = 0; q < NB; ++q)
                    if (q - KL == (int)k) w[q] = __fma_rn(vp, a, w[q]);
            }
        }
    }
}

// Build the coefficients for rows s .. s+R-1 of operator `op` (every thread
// of the group), then keep them in registers or write them to the table.
template <class C>
__device__ __forceinline__ void jw_prologue(const JwOperator& op, GroupCtx& g, int64_t s, JwCoef<C>& cf,
                                            double* table = nullptr)
{
    constexpr int R = C::kR;
    using S = typename JwCoef<C>::S;
    const int64_t M = op.M;
    double w[C::NB][R];
    // (1) effective matvec weights of V*A for each row
#pragma unroll
    for (int j = 0; j < R; ++j) {
        double wr[C::NB];
        if (s + j < M) {
            jw_row_weights<C::kKL, C::NB>(op, s + j, wr);
        } else {
#pragma unroll
            for (int k = 0; k < C::NB; ++k) wr[k] = 0.0;
        }
#pragma unroll
        for (int k = 0; k < C::NB; ++k) w[k][j] = wr[k];
    }
    // (2) solve coefficients in FP64
    double l64[R], h64[R], m64[R], a64[R], c64[R];
#pragma unroll
    for (int j = 0; j < R; ++j) { l64[j] = 0.0; h64[j] = 0.0; m64[j] = 1.0; a64[j] = 0.0; c64[j] = 0.0; }
    if constexpr (C::kSV == SV_TRI) {
        // Moebius product of this chunk: v_i = [[1, -a_i c_{i-1}], [1, 0]] v_{i-1}
        double a = 1, b = 0, c = 0, d = 1;
        double acs[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int64_t i = s + j;
            double ac = 0.0;
            if (i >= 1 && i < M) {
                const double ai = band(op, op.off_sl, i);
                const double cim1 = (i - 1 < M - 1) ? band(op, op.off_su, i - 1) : 0.0;
                ac = ai * cim1;
            }
            acs[j] = ac;
            const double na = a - ac * c, nb = b - ac * d;
            c = a; d = b; a = na; b = nb;
            renorm2x2(a, b, c, d);
        }
        group_matrix_scan(g, a, b, c, d);
        // incoming vector = Q * (1, 0)^T = (a, c): d'_{s-1} = a / c
        double dprev = (s == 0) ? 1.0 : a / c;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int64_t i = s + j;
            const double dp = (i == 0) ? 1.0 : 1.0 - acs[j] / dprev;
            const double dinv = 1.0 / dp;
            dprev = dp;
            const double ai = (i >= 1 && i < M) ? band(op, op.off_sl, i) : 0.0;
            const double ci = (i < M - 1) ? band(op, op.off_su, i) : 0.0;
            l64[j] = ai * dinv;
            h64[j] = ci * dinv;
            m64[j] = dinv;
            a64[j] = ai;
            c64[j] = ci;
        }
    } else if constexpr (C::kSV == SV_LOWER) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int64_t i = s + j;
            l64[j] = (i >= 1 && i < M) ? band(op, op.off_sl, i) : 0.0;
            a64[j] = l64[j];
        }
    } else if constexpr (C::kSV == SV_UPPER) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int64_t i = s + j;
            h64[j] = (i < M - 1) ? band(op, op.off_su, i) : 0.0;
            c64[j] = h64[j];
        }
    }
    if constexpr (!C::kMixed) {
#pragma unroll
        for (int j = 0; j < R; ++j)
#pragma unroll
            for (int k = 0; k < C::NB; ++k) w[k][j] *= m64[j];
    }
    double sc[R];
#pragma unroll
    for (int j = 0; j < R; ++j) sc[j] = C::kScale ? scale_factor(op.scale_kind, s + j, op.lshift, op.scale_s) : 1.0;
    if constexpr (C::kTbl) {
        const int T = cf.T, tt = cf.tt;
#pragma unroll
        for (int j = 0; j < R; ++j) {
#pragma unroll
            for (int k = 0; k < C::NB; ++k) table[(k * R + j) * T + tt] = w[k][j];
            if constexpr (C::kFwd) table[(C::P_L * R + j) * T + tt] = l64[j];
            if constexpr (C::kBwd) table[(C::P_H * R + j) * T + tt] = h64[j];
            if constexpr (C::kScale) table[(C::P_SC * R + j) * T + tt] = sc[j];
        }
    } else {
#pragma unroll
        for (int j = 0; j < R; ++j) {
#pragma unroll
            for (int k = 0; k < C::NB; ++k) cf.w_[k][j] = w[k][j];
            if constexpr (C::kFwd) cf.l_[j] = (S)l64[j];
            if constexpr (C::kBwd) cf.h_[j] = (S)h64[j];
            if constexpr (C::kScale) cf.sc_[j] = sc[j];
            if constexpr (C::kMixed) {
                cf.m_[j] = (S)m64[j];
                if constexpr (C::kFwd) cf.al_[j] = a64[j];
                if constexpr (C::kBwd) cf.cu_[j] = c64[j];
            }
        }
    }
}

// ---- Global <-> shared movement of one warp segment.
template <class C>
__device__ __forceinline__ void issue_segment_load(const JwIO& io, int64_t sys, int64_t r0, int lane,
                                                   typename C::TS* buf)
{
    using T = typename C::T;
    constexpr int R = C::kR, KL = C::kKL, KU = C::kKU;
    const int64_t M = io.M;
    const T* in = reinterpret_cast<const T*>(io.in);
    auto row_ok = [&](int64_t row) { return row >= 0 && row < M && row >= io.iz0 && row < io.iz1; };
    if constexpr (C::kLIN == LAY_REAL) {
        // ALT: row e of system sys is row 2 e + (sys & 1) of row set sys / 2
        const int64_t h = io.alt ? (sys & 1) : 0, es = io.alt ? 2 : 1;
        const int64_t Msys = io.alt ? (M - h + 1) >> 1 : M;
        auto ok_at = [&](int64_t e) { return e >= 0 && e < Msys && row_ok(es * e + h); };
        const T* base = in + io.in_off + (io.alt ? sys >> 1 : sys) * io.in_stride + h;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int q = 32 * k + lane;
            const int64_t row = r0 + q;
            const bool ok = ok_at(row);
            cp_async_elem<T>(buf + swz<R, false>(q), ok ? base + es * row : in, ok);
        }
        if (KL > 0 && lane < KL) {
            const int64_t row = r0 - KL + lane;
            const bool ok = ok_at(row);
            cp_async_elem<T>(buf + 32 * R + lane, ok ? base + es * row : in, ok);
        }
        if (KU > 0 && lane < KU) {
            const int64_t row = r0 + 32 * R + lane;
            const bool ok = ok_at(row);
            cp_async_elem<T>(buf + 32 * R + KL + lane, ok ? base + es * row : in, ok);
        }
    } else {  // XXII complex: real part row block 2*sys, imaginary 2*sys+1
        const T* re = in + io.in_off + (2 * sys) * io.in_stride;
        const T* im = re + io.in_stride;
        auto put = [&](int slot, int64_t row) {
            const bool ok = row_ok(row);
            T* dst = reinterpret_cast<T*>(buf + slot);
            cp_async_elem<T>(dst, ok ? re + row : in, ok);
            cp_async_elem<T>(dst + 1, ok ? im + row : in, ok);
        };
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int q = 32 * k + lane;
            put(swz<R, true>(q), r0 + q);
        }
        if (KL > 0 && lane < KL) put(32 * R + lane, r0 - KL + lane);
        if (KU > 0 && lane < KU) put(32 * R + KL + lane, r0 + 32 * R + lane);
    }
}

template <class C>
__device__ __forceinline__ void store_segment(const JwIO& io, int64_t sys, int64_t r0, int lane,
                                              const typename C::TS* buf)
{
    using T = typename C::T;
    using T2 = typename Vec2Of<T>::type;
    constexpr int R = C::kR;
    T* out = reinterpret_cast<T*>(io.out);
    const int64_t M = io.M;
    const int64_t h = io.alt ? (sys & 1) : 0, es = io.alt ? 2 : 1;
    const int64_t Msys = io.alt ? (M - h + 1) >> 1 : M;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int q = 32 * k + lane;
        const int64_t row = r0 + q;
        if (row >= Msys || es * row + h < io.oz0 || es * row + h >= io.oz1) continue;
        if constexpr (C::kLOUT == LAY_REAL) {
            T v = buf[swz<R, false>(q)];
            T* p = out + io.out_off + (io.alt ? sys >> 1 : sys) * io.out_stride + es * row + h;
            if (io.accumulate) v += *p;
            *p = v;
        } else if constexpr (C::kLOUT == LAY_PACKED) {
            T2 v = buf[swz<R, true>(q)];
            T2* p = reinterpret_cast<T2*>(io.out) + io.out_off + sys * io.out_stride + row;
            if (io.accumulate) {
                const T2 o = *p;
                v.x += o.x;
                v.y += o.y;
            }
            *p = v;
        } else {  // XXII complex output
            T2 v = buf[swz<R, true>(q)];
            T* pr = out + io.out_off + (2 * sys) * io.out_stride + row;
            T* pi = pr + io.out_stride;
            if (io.accumulate) {
                v.x += *pr;
                v.y += *pi;
            }
            *pr = v.x;
            *pi = v.y;
        }
    }
}

// ---- Unit-diagonal solve of one chunk.
// Forward: z_j = x_j - l_j z_{j-1}; backward: x_j = z_j - h_j x_{j+1}.  The
// chunk-boundary couplings go through the affine scans; the in-chunk products
// F_j = prod_{k<=j}(-l_k) and G_j = prod_{k>=j}(-h_k) are rebuilt on the fly.
template <int R, int SV, class V, class S, class LF, class HF>
__device__ __forceinline__ void chunk_solve(GroupCtx& g, LF lget, HF hget, V (&x)[R])
{
    using O = VOps<V>;
    constexpr bool FWD = (SV == SV_LOWER || SV == SV_TRI);
    constexpr bool BWD = (SV == SV_UPPER || SV == SV_TRI);
    if constexpr (FWD) {
        // in place: x holds z after the local forward pass
        S A = -lget(0);
#pragma unroll
        for (int j = 1; j < R; ++j) {
            const S lj = lget(j);
            x[j] = O::fma(-lj, x[j - 1], x[j]);
            A = -lj * A;
        }
        const V pin = group_affine_scan<V, S, true>(g, A, x[R - 1]);
        S p = S(1);
#pragma unroll
        for (int j = 0; j < R; ++j) {
            p = -lget(j) * p;
            x[j] = O::fma(p, pin, x[j]);
        }
    }
    if constexpr (SV == SV_UPPER || SV == SV_TRI) {
#pragma unroll
        for (int j = R - 2; j >= 0; --j) x[j] = O::fma(-hget(j), x[j + 1], x[j]);
    }
    if constexpr (BWD) {
        S Ab = S(1);
#pragma unroll
        for (int j = 0; j < R; ++j) Ab = -hget(j) * Ab;
        const V q = group_affine_scan<V, S, false>(g, Ab, x[0]);
        S p = S(1);
#pragma unroll
        for (int j = R - 1; j >= 0; --j) {
            p = -hget(j) * p;
            x[j] = O::fma(p, q, x[j]);
        }
    }
}

// Mixed precision: x = M^{-1} g with FP32 solves and FP64 residuals
// (`sweeps` FP32 solves: one initial, sweeps-1 refinements).
template <class C>
__device__ __forceinline__ void mixed_solve(GroupCtx& g, const JwCoef<C>& cf, int sweeps, typename C::V (&x)[C::kR])
{
    using V = typename C::V;
    using VF = typename C::VF;
    using O = VOps<V>;
    using OF = VOps<VF>;
    constexpr int R = C::kR, SV = C::kSV;
    V gv[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
        gv[j] = x[j];
        x[j] = O::zero();
    }
    for (int it = 0; it < sweeps; ++it) {
        V r[R];
        if (it == 0) {
#pragma unroll
            for (int j = 0; j < R; ++j) r[j] = gv[j];
        } else {
            V prev, next;
            group_neighbours<V>(g, x[0], x[R - 1], prev, next);
#pragma unroll
            for (int j = 0; j < R; ++j) {
                V mx = x[j];
                if constexpr (C::kFwd) mx = O::fma(cf.al_[j], j > 0 ? x[j - 1] : prev, mx);
                if constexpr (C::kBwd) mx = O::fma(cf.cu_[j], j < R - 1 ? x[j + 1] : next, mx);
                r[j] = O::fma(-1.0, mx, gv[j]);
            }
        }
        VF d[R];
#pragma unroll
        for (int j = 0; j < R; ++j) d[j] = OF::mul(cf.m_[j], to_f32(r[j]));
        chunk_solve<R, SV, VF, float>(g, [&](int j) { return cf.l_[j]; }, [&](int j) { return cf.h_[j]; }, d);
#pragma unroll
        for (int j = 0; j < R; ++j) x[j] = O::add(x[j], to_f64(d[j]));
    }
}

// ---- Process systems sys0, sys0+step, ... with the group's coefficients.
template <class C>
__device__ __forceinline__ void jw_run_systems(const JwOperator& op, const JwIO& io, GroupCtx& g,
                                               const JwCoef<C>& cf, typename C::TS* buf0, typename C::TS* buf1,
                                               int64_t sys0, int64_t step)
{
    using V = typename C::V;
    using TS = typename C::TS;
    using O = VOps<V>;
    constexpr int R = C::kR, KL = C::kKL, KU = C::kKU;
    constexpr bool CPLX = C::kCplx;
    const int64_t r0 = (int64_t)g.wg * 32 * R;
    const int64_t s = r0 + (int64_t)g.lane * R;
    if (sys0 >= io.nsys) return;
    issue_segment_load<C>(io, sys0, r0, g.lane, buf0);
    cp_async_commit();
    int it = 0;
    for (int64_t sys = sys0; sys < io.nsys; sys += step, ++it) {
        TS* cur = (it & 1) ? buf1 : buf0;
        TS* nxt = (it & 1) ? buf0 : buf1;
        if (sys + step < io.nsys) issue_segment_load<C>(io, sys + step, r0, g.lane, nxt);
        cp_async_commit();
        cp_async_wait<1>();
        __syncwarp();
        // In place, a warp's halo rows belong to its neighbour warps: every
        // warp of the group must hold this system's input before any warp
        // stores results.  Solves get that ordering from their scan barriers.
        if constexpr (C::kSV == SV_NONE && (KL + KU) > 0) {
            if (g.W > 1) group_bar(g.bar_id, g.nthr);
        }
        // chunk rows s-KL .. s+R+KU-1
        V be[R + KL + KU];
#pragma unroll
        for (int j = 0; j < R + KL + KU; ++j) {
            const int q = g.lane * R + j - KL;
            int slot;
            if (q < 0) slot = 32 * R + (q + KL);
            else if (q >= 32 * R) slot = 32 * R + KL + (q - 32 * R);
            else slot = swz<R, CPLX>(q);
            be[j] = conv<V>(cur[slot]);
        }
        V x[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            V acc = O::mul(cf.w(0, j), be[j]);
#pragma unroll
            for (int k = 1; k < C::NB; ++k) acc = O::fma(cf.w(k, j), be[j + k], acc);
            x[j] = acc;
        }
        if constexpr (C::kMixed) {
            mixed_solve<C>(g, cf, op.refine_sweeps, x);
        } else if constexpr (C::kSV != SV_NONE) {
            chunk_solve<R, C::kSV, V, typename JwCoef<C>::S>(g, [&](int j) { return cf.l(j); },
                                                             [&](int j) { return cf.h(j); }, x);
        }
        if (C::kSV != SV_NONE && s == 0) x[0] = O::mul(op.scaleC, x[0]);
        if constexpr (C::kScale) {
#pragma unroll
            for (int j = 0; j < R; ++j) x[j] = O::mul(cf.sc(j), x[j]);
        }
        __syncwarp();  // every lane has read `cur`
#pragma unroll
        for (int j = 0; j < R; ++j) cur[swz<R, CPLX>(g.lane * R + j)] = conv<TS>(x[j]);
        __syncwarp();
        store_segment<C>(io, sys, r0, g.lane, cur);
        __syncwarp();  // `cur` is the target of the load issued next iteration
    }
    cp_async_wait<0>();
}

template <class C>
__global__ void __launch_bounds__(C::kMaxThreads) jw_step_kernel(const JwOperator op, const JwIO io, const int W)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using TS = typename C::TS;
    const int warp = threadIdx.x >> 5;
    const int G = blockDim.x / (32 * W);
    const int grp = warp / W;
    GroupCtx g;
    g.lane = threadIdx.x & 31;
    g.wg = warp - grp * W;
    g.W = W;
    g.nthr = 32 * W;
    g.bar_id = 1 + grp;
    g.seq = 0;
    constexpr size_t per_warp = jw_smem_per_warp<C>();
    double* table = reinterpret_cast<double*>(smem_raw);
    unsigned char* data = smem_raw + jw_table_bytes<C>(W);
    TS* buf0 = reinterpret_cast<TS*>(data + (size_t)warp * per_warp);
    TS* buf1 = buf0 + C::SEG;
    g.scratch = reinterpret_cast<double*>(data + (size_t)G * W * per_warp) + (size_t)grp * W * kScratchPerWarp;

    const int64_t s = (int64_t)(g.wg * 32 + g.lane) * C::kR;
    JwCoef<C> cf;
    cf.tbl = table;
    cf.T = 32 * W;
    cf.tt = g.wg * 32 + g.lane;
    const int64_t sys0 = (int64_t)blockIdx.x * G + grp;
    const int64_t step = (int64_t)gridDim.x * G;
    // ALT: this group's systems all have the parity of sys0 (the launch makes
    // the system step even); the odd rows' system has no scaleC row
    JwOperator opg = op;
    if (op.alt) {
        opg.alt_h = (int)(sys0 & 1);
        opg.M = (op.M - opg.alt_h + 1) >> 1;
        if (opg.alt_h) opg.scaleC = 1.0;
    }
    if constexpr (C::kTbl) {
        // every group of the CTA solves with the same matrix: group 0 builds
        // the shared table once (not used in ALT mode)
        if (grp == 0) jw_prologue<C>(opg, g, s, cf, table);
        __syncthreads();
    } else {
        jw_prologue<C>(opg, g, s, cf);
    }
    jw_run_systems<C>(opg, io, g, cf, buf0, buf1, sys0, step);
}

// ---- Uneven batch: one persistent launch over many matrices of different
// sizes.  Each group takes (entry, system range) items from a global counter
// (largest items first), refactors when the entry changes and streams the
// item's systems.  Item fetch: the group leader's atomicAdd is broadcast
// through two alternating shared slots, one barrier per fetch.
template <class C>
__global__ void __launch_bounds__(256) jw_batch_kernel(const BatchEntryDev* __restrict__ entries,
                                                      const WorkItem* __restrict__ items, const int nitems,
                                                      unsigned int* __restrict__ counter, const int W)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using TS = typename C::TS;
    const int warp = threadIdx.x >> 5;
    const int G = blockDim.x / (32 * W);
    const int grp = warp / W;
    GroupCtx g;
    g.lane = threadIdx.x & 31;
    g.wg = warp - grp * W;
    g.W = W;
    g.nthr = 32 * W;
    g.bar_id = 1 + grp;
    g.seq = 0;
    constexpr size_t per_warp = jw_smem_per_warp<C>();
    TS* buf0 = reinterpret_cast<TS*>(smem_raw + (size_t)warp * per_warp);
    TS* buf1 = buf0 + C::SEG;
    double* scratch_all = reinterpret_cast<double*>(smem_raw + (size_t)G * W * per_warp);
    g.scratch = scratch_all + (size_t)grp * W * kScratchPerWarp;
    int* slots = reinterpret_cast<int*>(scratch_all + (size_t)G * W * kScratchPerWarp) + 2 * grp;
    const int64_t s = (int64_t)(g.wg * 32 + g.lane) * C::kR;

    JwCoef<C> cf;
    int cur_entry = -1;
    int par = 0;
    for (;;) {
        int it = 0;
        if (W == 1) {
            if (g.lane == 0) it = (int)atomicAdd(counter, 1u);
            it = __shfl_sync(FULL, it, 0);
        } else {
            if (g.wg == 0 && g.lane == 0) slots[par] = (int)atomicAdd(counter, 1u);
            __syncwarp();
            group_bar(g.bar_id, g.nthr);
            it = slots[par];
            par ^= 1;
        }
        if (it >= nitems) break;
        const WorkItem wi = items[it];
        const JwOperator op = entries[wi.entry].op;
        JwIO io = entries[wi.entry].io;
        io.nsys = wi.y1;
        if (wi.entry != cur_entry) {
            jw_prologue<C>(op, g, s, cf);
            cur_entry = wi.entry;
        }
        jw_run_systems<C>(op, io, g, cf, buf0, buf1, wi.y0, 1);
    }
}

template <class C>
__host__ size_t jw_batch_smem_bytes(int W, int G)
{
    return jw_smem_bytes<C>(W, G) + (size_t)G * 2 * sizeof(int);
}

}  // namespace pfb
