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
#pragma once
#include "common.cuh"
#include "jw_types.h"

namespace pfb {

template <int R, int KL, int KU, int SV, int LIN, int LOUT, bool SCALE>
struct JwCfg {
    static constexpr int kR = R, kKL = KL, kKU = KU, kSV = SV, kLIN = LIN, kLOUT = LOUT;
    static constexpr bool kScale = SCALE;
    static constexpr bool kCplx = (LIN != LAY_REAL);
    using V = typename std::conditional<kCplx, double2, double>::type;
    static constexpr int NB = KL + KU + 1;
    static constexpr int SEG = 32 * R + KL + KU;  // elements per warp buffer
    static constexpr bool kFwd = (SV == SV_LOWER || SV == SV_TRI);
    static constexpr bool kBwd = (SV == SV_UPPER || SV == SV_TRI);
};

// Shared memory per warp: two segment buffers (16-byte aligned).  The scan
// scratch (16 doubles per warp) follows all warp buffers.
template <class C>
__host__ __device__ constexpr size_t jw_smem_per_warp()
{
    return ((2 * (size_t)C::SEG * sizeof(typename C::V)) + 15) / 16 * 16;
}

__device__ __forceinline__ int64_t band_pos(const JwOperator& op, int64_t i)
{
    if (!op.perm) return i;
    int64_t t = i / op.perm_r, j = i - t * op.perm_r;
    return t + ((j < op.perm_m) ? j * op.perm_ceil : op.perm_m * op.perm_ceil + (j - op.perm_m) * op.perm_floor);
}

__device__ __forceinline__ double band(const JwOperator& op, int64_t off, int64_t i)
{
    return __ldg(op.bands + off + band_pos(op, i));
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

// Per-thread coefficients of one matrix.
template <class C>
struct JwCoef {
    double w[C::NB][C::kR];  // matvec weights, offsets -KL..KU, solve scaling folded in
    double l[C::kFwd ? C::kR : 1];
    double F[C::kFwd ? C::kR : 1];
    double h[C::kBwd ? C::kR : 1];
    double G[C::kBwd ? C::kR : 1];
    double sc[C::kScale ? C::kR : 1];
};

// Scan scratch: 16 doubles per warp, [direction*8 + parity*4 + {A, -, B.x, B.y}].
// Alternating the parity per system keeps a fast warp from overwriting an
// aggregate a slower warp of the same group has not read yet.
struct GroupCtx {
    int lane, wg, W, nthr, bar_id, par;
    double* scratch;  // scratch of warp 0 of this group; warp w at scratch + 16*w
};

// Exclusive scan of affine maps y = B + A*x over the group, in row order
// (forward) or reverse row order (backward).  Returns the incoming value of
// this thread.  `in0` is the value entering the first (last) thread.
template <class V, bool FORWARD>
__device__ __forceinline__ V group_affine_scan(const GroupCtx& g, double A, V B)
{
    using O = VOps<V>;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        double Ap = FORWARD ? __shfl_up_sync(FULL, A, d) : __shfl_down_sync(FULL, A, d);
        V Bp = FORWARD ? O::shfl_up(B, d) : O::shfl_down(B, d);
        bool take = FORWARD ? (g.lane >= d) : (g.lane + d < 32);
        if (take) {
            B = O::fma(A, Bp, B);
            A = A * Ap;
        }
    }
    // exclusive map of this lane within its warp
    double Ae = FORWARD ? __shfl_up_sync(FULL, A, 1) : __shfl_down_sync(FULL, A, 1);
    V Be = FORWARD ? O::shfl_up(B, 1) : O::shfl_down(B, 1);
    const bool first = FORWARD ? (g.lane == 0) : (g.lane == 31);
    if (first) {
        Ae = 1.0;
        Be = O::zero();
    }
    V win = O::zero();
    if (g.W > 1) {
        // warp aggregate = inclusive map of the warp's last (first) lane
        const int slot = (FORWARD ? 0 : 8) + 4 * g.par;
        double* my = g.scratch + 16 * g.wg + slot;
        const bool agg = FORWARD ? (g.lane == 31) : (g.lane == 0);
        if (agg) {
            my[0] = A;
            *reinterpret_cast<V*>(my + 2) = B;
        }
        __syncwarp();
        group_bar(g.bar_id, g.nthr);
        if (FORWARD) {
            for (int w = 0; w < g.wg; ++w) {
                const double* o = g.scratch + 16 * w + slot;
                win = O::fma(o[0], win, *reinterpret_cast<const V*>(o + 2));
            }
        } else {
            for (int w = g.W - 1; w > g.wg; --w) {
                const double* o = g.scratch + 16 * w + slot;
                win = O::fma(o[0], win, *reinterpret_cast<const V*>(o + 2));
            }
        }
    }
    return O::fma(Ae, win, Be);
}

// Exclusive scan of 2x2 matrix products P_t * ... * P_0 (row order) used by
// the tridiagonal factorisation.  Returns the product of all preceding chunks.
__device__ __forceinline__ void group_matrix_scan(const GroupCtx& g, double& a, double& b, double& c, double& d)
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
        double* my = g.scratch + 16 * g.wg;
        if (g.lane == 31) { my[0] = a; my[1] = b; my[2] = c; my[3] = d; }
        __syncwarp();
        group_bar(g.bar_id, g.nthr);
        for (int w = 0; w < g.wg; ++w) {
            const double* o = g.scratch + 16 * w;
            double na = o[0] * wa + o[1] * wc, nb = o[0] * wb + o[1] * wd;
            double nc = o[2] * wa + o[3] * wc, nd = o[2] * wb + o[3] * wd;
            wa = na; wb = nb; wc = nc; wd = nd;
            renorm2x2(wa, wb, wc, wd);
        }
        group_bar(g.bar_id, g.nthr);  // scratch is reused by the next scan
    }
    a = ea * wa + eb * wc;
    b = ea * wb + eb * wd;
    c = ec * wa + ed * wc;
    d = ec * wb + ed * wd;
}

// Build the per-thread coefficients for rows s .. s+R-1 of operator `op`.
template <class C>
__device__ __forceinline__ void jw_prologue(const JwOperator& op, const GroupCtx& g, int64_t s, JwCoef<C>& cf)
{
    constexpr int R = C::kR, KL = C::kKL, KU = C::kKU;
    const int64_t M = op.M;
    // (1) effective matvec weights of V*A for each row
#pragma unroll
    for (int j = 0; j < R; ++j) {
#pragma unroll
        for (int k = 0; k < C::NB; ++k) cf.w[k][j] = 0.0;
        const int64_t i = s + j;
        if (i < M) {
            double vl = 0, vd = 1, vu = 0;
            if (op.mvj != MVJ_NONE) vd = band(op, op.off_md, i);
            if (op.mvj == MVJ_UPPER && i + 1 < M) vu = band(op, op.off_mo, i);
            if (op.mvj == MVJ_LOWER && i >= 1) vl = band(op, op.off_mo, i);
            if (op.dgbmv == nullptr) {
                if constexpr (KL >= 1) cf.w[KL - 1][j] = vl;
                cf.w[KL][j] = vd;
                if constexpr (KU >= 1) cf.w[KL + 1][j] = vu;
            } else {
                const int kla = op.dg_lda - 1 - op.dg_ku;
                for (int pv = -1; pv <= 1; ++pv) {
                    const double vp = (pv < 0) ? vl : (pv == 0 ? vd : vu);
                    const int64_t p = i + pv;
                    if (vp == 0.0 || p < 0 || p >= M) continue;
                    for (int kk = -kla; kk <= op.dg_ku; ++kk) {
                        const int64_t c = p + kk;
                        if (c < 0 || c >= M) continue;
                        const double a = __ldg(op.dgbmv + op.dg_off + (int64_t)(op.dg_ku - kk) * M + c);
                        const int64_t k = c - i;  // within [-KL, KU] by construction of the plan
#pragma unroll
                        for (int q = 0; q < C::NB; ++q)
                            if (q - KL == (int)k) cf.w[q][j] = __fma_rn(vp, a, cf.w[q][j]);
                    }
                }
            }
        }
    }
    // (2) solve coefficients
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
            // [[1,-ac],[1,0]] * [[a,b],[c,d]]
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
            cf.l[j] = ai * dinv;
            cf.h[j] = ci * dinv;
#pragma unroll
            for (int k = 0; k < C::NB; ++k) cf.w[k][j] *= dinv;
        }
    } else if constexpr (C::kSV == SV_LOWER) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int64_t i = s + j;
            cf.l[j] = (i >= 1 && i < M) ? band(op, op.off_sl, i) : 0.0;
        }
    } else if constexpr (C::kSV == SV_UPPER) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int64_t i = s + j;
            cf.h[j] = (i < M - 1) ? band(op, op.off_su, i) : 0.0;
        }
    }
    if constexpr (C::kFwd) {
        double p = 1.0;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            p = -cf.l[j] * p;
            cf.F[j] = p;
        }
    }
    if constexpr (C::kBwd) {
        double p = 1.0;
#pragma unroll
        for (int j = R - 1; j >= 0; --j) {
            p = -cf.h[j] * p;
            cf.G[j] = p;
        }
    }
    if constexpr (C::kScale) {
#pragma unroll
        for (int j = 0; j < R; ++j) cf.sc[j] = scale_factor(op.scale_kind, s + j, op.lshift, op.scale_s);
    }
}

// ---- Global <-> shared movement of one warp segment.
template <class C>
__device__ __forceinline__ void issue_segment_load(const JwIO& io, int64_t sys, int64_t r0, int lane,
                                                   typename C::V* buf)
{
    constexpr int R = C::kR, KL = C::kKL, KU = C::kKU;
    const int64_t M = io.M;
    auto row_ok = [&](int64_t row) { return row >= 0 && row < M && row >= io.iz0 && row < io.iz1; };
    if constexpr (C::kLIN == LAY_REAL) {
        const double* base = io.in + io.in_off + sys * io.in_stride;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int q = 32 * k + lane;
            const int64_t row = r0 + q;
            const bool ok = row_ok(row);
            cp_async8(buf + swz<R, false>(q), ok ? base + row : io.in, ok);
        }
        if (KL > 0 && lane < KL) {
            const int64_t row = r0 - KL + lane;
            const bool ok = row_ok(row);
            cp_async8(buf + 32 * R + lane, ok ? base + row : io.in, ok);
        }
        if (KU > 0 && lane < KU) {
            const int64_t row = r0 + 32 * R + lane;
            const bool ok = row_ok(row);
            cp_async8(buf + 32 * R + KL + lane, ok ? base + row : io.in, ok);
        }
    } else {  // XXII complex: real part row block 2*sys, imaginary 2*sys+1
        const double* re = io.in + io.in_off + (2 * sys) * io.in_stride;
        const double* im = re + io.in_stride;
        auto put = [&](int slot, int64_t row) {
            const bool ok = row_ok(row);
            double* dst = reinterpret_cast<double*>(buf + slot);
            cp_async8(dst, ok ? re + row : io.in, ok);
            cp_async8(dst + 1, ok ? im + row : io.in, ok);
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
                                              const typename C::V* buf)
{
    constexpr int R = C::kR;
    const int64_t M = io.M;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int q = 32 * k + lane;
        const int64_t row = r0 + q;
        if (row >= M || row < io.oz0 || row >= io.oz1) continue;
        if constexpr (C::kLOUT == LAY_REAL) {
            double v = buf[swz<R, false>(q)];
            double* p = io.out + io.out_off + sys * io.out_stride + row;
            if (io.accumulate) v += *p;
            *p = v;
        } else if constexpr (C::kLOUT == LAY_PACKED) {
            double2 v = buf[swz<R, true>(q)];
            double2* p = reinterpret_cast<double2*>(io.out) + io.out_off + sys * io.out_stride + row;
            if (io.accumulate) {
                const double2 o = *p;
                v.x += o.x;
                v.y += o.y;
            }
            *p = v;
        } else {  // XXII complex output
            double2 v = buf[swz<R, true>(q)];
            double* pr = io.out + io.out_off + (2 * sys) * io.out_stride + row;
            double* pi = pr + io.out_stride;
            if (io.accumulate) {
                v.x += *pr;
                v.y += *pi;
            }
            *pr = v.x;
            *pi = v.y;
        }
    }
}

// ---- Solve one system whose chunk values are in x (after the matvec).
template <class C>
__device__ __forceinline__ void jw_solve_chunk(const GroupCtx& g, const JwCoef<C>& cf, typename C::V (&x)[C::kR])
{
    using V = typename C::V;
    using O = VOps<V>;
    constexpr int R = C::kR;
    if constexpr (C::kFwd) {
        V z[R];
        z[0] = x[0];
#pragma unroll
        for (int j = 1; j < R; ++j) z[j] = O::fma(-cf.l[j], z[j - 1], x[j]);
        const V pin = group_affine_scan<V, true>(g, cf.F[R - 1], z[R - 1]);
        if constexpr (C::kSV == SV_LOWER) {
#pragma unroll
            for (int j = 0; j < R; ++j) x[j] = O::fma(cf.F[j], pin, z[j]);
        } else {
            x[R - 1] = O::fma(cf.F[R - 1], pin, z[R - 1]);
#pragma unroll
            for (int j = R - 2; j >= 0; --j) x[j] = O::fma(-cf.h[j], x[j + 1], O::fma(cf.F[j], pin, z[j]));
        }
    } else if constexpr (C::kSV == SV_UPPER) {
#pragma unroll
        for (int j = R - 2; j >= 0; --j) x[j] = O::fma(-cf.h[j], x[j + 1], x[j]);
    }
    if constexpr (C::kBwd) {
        const V q = group_affine_scan<V, false>(g, cf.G[0], x[0]);
#pragma unroll
        for (int j = 0; j < R; ++j) x[j] = O::fma(cf.G[j], q, x[j]);
    }
}

// ---- Process systems sys0, sys0+step, ... with the group's coefficients.
template <class C>
__device__ __forceinline__ void jw_run_systems(const JwOperator& op, const JwIO& io, GroupCtx g,
                                               const JwCoef<C>& cf, typename C::V* buf0, typename C::V* buf1,
                                               int64_t sys0, int64_t step)
{
    using V = typename C::V;
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
        g.par = it & 1;
        V* cur = (it & 1) ? buf1 : buf0;
        V* nxt = (it & 1) ? buf0 : buf1;
        if (sys + step < io.nsys) issue_segment_load<C>(io, sys + step, r0, g.lane, nxt);
        cp_async_commit();
        cp_async_wait<1>();
        __syncwarp();
        // chunk rows s-KL .. s+R+KU-1
        V be[R + KL + KU];
#pragma unroll
        for (int j = 0; j < R + KL + KU; ++j) {
            const int q = g.lane * R + j - KL;
            int slot;
            if (q < 0) slot = 32 * R + (q + KL);
            else if (q >= 32 * R) slot = 32 * R + KL + (q - 32 * R);
            else slot = swz<R, CPLX>(q);
            be[j] = cur[slot];
        }
        V x[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            V acc = O::mul(cf.w[0][j], be[j]);
#pragma unroll
            for (int k = 1; k < C::NB; ++k) acc = O::fma(cf.w[k][j], be[j + k], acc);
            x[j] = acc;
        }
        jw_solve_chunk<C>(g, cf, x);
        if (C::kSV != SV_NONE && s == 0) x[0] = O::mul(op.scaleC, x[0]);
        if constexpr (C::kScale) {
#pragma unroll
            for (int j = 0; j < R; ++j) x[j] = O::mul(cf.sc[j], x[j]);
        }
        __syncwarp();  // every lane has read `cur`
#pragma unroll
        for (int j = 0; j < R; ++j) cur[swz<R, CPLX>(g.lane * R + j)] = x[j];
        __syncwarp();
        store_segment<C>(io, sys, r0, g.lane, cur);
        __syncwarp();  // `cur` is the target of the load issued next iteration
    }
    cp_async_wait<0>();
}

template <class C>
__global__ void __launch_bounds__(256) jw_step_kernel(const JwOperator op, const JwIO io, const int W)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using V = typename C::V;
    const int warp = threadIdx.x >> 5;
    const int G = blockDim.x / (32 * W);
    const int grp = warp / W;
    GroupCtx g;
    g.lane = threadIdx.x & 31;
    g.wg = warp - grp * W;
    g.W = W;
    g.nthr = 32 * W;
    g.bar_id = 1 + grp;
    g.par = 0;
    constexpr size_t per_warp = jw_smem_per_warp<C>();
    V* buf0 = reinterpret_cast<V*>(smem_raw + (size_t)warp * per_warp);
    V* buf1 = buf0 + C::SEG;
    g.scratch = reinterpret_cast<double*>(smem_raw + (size_t)G * W * per_warp) + (size_t)grp * W * 16;

    const int64_t s = (int64_t)(g.wg * 32 + g.lane) * C::kR;
    JwCoef<C> cf;
    jw_prologue<C>(op, g, s, cf);
    const int64_t sys0 = (int64_t)blockIdx.x * G + grp;
    const int64_t step = (int64_t)gridDim.x * G;
    jw_run_systems<C>(op, io, g, cf, buf0, buf1, sys0, step);
}

template <class C>
__host__ size_t jw_smem_bytes(int W, int G)
{
    return (size_t)G * W * jw_smem_per_warp<C>() + (size_t)G * W * 16 * sizeof(double);
}

}  // namespace pfb
