// jw_steps.cuh -- K consecutive JW steps in one kernel (numConsecutiveJWIterations).
//
// The reference generates one kernel that keeps a right-hand side in registers
// for K order-changing steps (PfSolve/pfSolve_CodeGen/pfSolve_KernelsLevel2/
// pfSolve_JonesWorland.h:108-374): step s works on M_s = M - s rows
// (upperBanded 1, 2) or M + s rows (upperBanded 0), with its own bands (buffer
// s of useMultipleInputBuffers, else buffer 0 at offsets that depend on M_s),
// the matvec diagonal applied at the first (upperBanded 1) or last
// (upperBanded 0) step only, and scaleC on solution row 0 after every solve.
// Rows at or beyond M_s pass through a step unchanged; the result is written
// for the final M_{K-1} rows only.
//
// Design:
//  * A group of W warps owns one system at a time; thread t owns rows
//    [R t, R t + R) for all K steps, so the data crosses HBM once per system
//    (read M rows, write M_{K-1} rows) however many steps run.
//  * The coefficients of every step -- matvec weights with the tridiagonal
//    pivots folded in, and the solve's l and h -- are built once per CTA into
//    a shared table (K x planes x rows doubles, read as 16-byte pairs) shared
//    by all groups of the CTA.  The pivots of each step come from the Moebius
//    scan of the group kernel's prologue.
//  * Per step: neighbour rows for the matvec by warp shuffles (shared memory
//    across warps), the unit-diagonal solve by the group kernel's chunk solve
//    (in-register recurrences + affine scans).
//  * Right-hand sides are read and written straight from registers (16-byte
//    accesses when the rows are 16-byte aligned), the next system's rows are
//    loaded while the current one is solved.
#pragma once
#include "jw_kernel.cuh"

namespace pfb {

template <int R_, int KL_, int KU_, int SV_, bool MV_>
struct KsCfg {
    static constexpr int R = R_, KL = KL_, KU = KU_, SV = SV_;
    static constexpr bool MV = MV_;
    static constexpr int NB = KL + KU + 1;
    static constexpr bool FWD = (SV == SV_LOWER || SV == SV_TRI);
    static constexpr bool BWD = (SV == SV_UPPER || SV == SV_TRI);
    // planes per step: NB weights, l (forward solves), h (backward solves)
    static constexpr int P_L = NB, P_H = NB + (FWD ? 1 : 0);
    static constexpr int NPL = P_H + (BWD ? 1 : 0);
    static constexpr int U = R / 2;
    // 16 rows per thread need more than the 128 registers of 512-thread CTAs
    static constexpr int kMaxThreads = R >= 16 ? 256 : 512;
    static_assert(R % 2 == 0 && R >= 2 && R <= 16, "rows per thread");
};

template <class C>
__host__ __device__ constexpr size_t ks_table_bytes(int K, int T)
{
    return (size_t)K * C::NPL * C::R * T * sizeof(double);
}

template <class C>
__host__ __device__ constexpr size_t ks_smem_bytes(int K, int W, int G)
{
    return ks_table_bytes<C>(K, 32 * W) + (size_t)G * W * kScratchPerWarp * sizeof(double);
}

__device__ __forceinline__ double step_band(const JwSteps& S, const JwStepDesc& d, int64_t off, int64_t i)
{
    int64_t pos = i;
    if (S.perm) {
        const int64_t t = i / d.perm_r, j = i - t * d.perm_r;
        pos = t + ((j < d.perm_m) ? j * d.perm_ceil : d.perm_m * d.perm_ceil + (j - d.perm_m) * d.perm_floor);
    }
    return __ldg(d.bands + off + pos);
}

// ---- Table of every step, built by all threads of the CTA: plane p of step
// s, rows 2u and 2u+1 of thread tt at ((s*NPL + p)*U + u)*T + tt (double2).
template <class C>
__device__ void ks_prologue(const JwSteps& S, double2* table, double* scratch, int T)
{
    constexpr int R = C::R, U = C::U, KL = C::KL, KU = C::KU;
    const int rows = R * T;
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int Rp = (rows + nthr - 1) / nthr;
    const int64_t s0 = (int64_t)tid * Rp;
    GroupCtx g;
    g.lane = tid & 31;
    g.wg = tid >> 5;
    g.W = nthr >> 5;
    g.nthr = nthr;
    g.bar_id = 1;
    g.seq = 0;
    g.scratch = scratch;
    double* tb = reinterpret_cast<double*>(table);
    for (int s = 0; s < S.K; ++s) {
        const JwStepDesc& d = S.st[s];
        const int64_t Ms = d.M;
        double dprev = 1.0;
        if constexpr (C::SV == SV_TRI) {
            double a = 1, b = 0, c = 0, dd = 1;
            for (int j = 0; j < Rp; ++j) {
                const int64_t i = s0 + j;
                double ac = 0.0;
                if (i >= 1 && i < Ms) ac = step_band(S, d, d.off_sl, i) * step_band(S, d, d.off_su, i - 1);
                const double na = a - ac * c, nb = b - ac * dd;
                c = a;
                dd = b;
                a = na;
                b = nb;
                renorm2x2(a, b, c, dd);
            }
            group_matrix_scan(g, a, b, c, dd);
            dprev = (s0 == 0) ? 1.0 : a / c;
        }
        for (int j = 0; j < Rp; ++j) {
            const int64_t i = s0 + j;
            if (i >= rows) break;
            double w[C::NB];
#pragma unroll
            for (int k = 0; k < C::NB; ++k) w[k] = 0.0;
            w[KL] = 1.0;
            double l = 0.0, h = 0.0;
            if (i < Ms) {
                if constexpr (C::MV) {
                    if (d.diag) w[KL] = step_band(S, d, d.off_md, i);
                    if constexpr (KU > 0) w[KL + 1] = step_band(S, d, d.off_mo, i);
                    if constexpr (KL > 0) w[KL - 1] = (i >= 1) ? step_band(S, d, d.off_mo, i) : 0.0;
                }
                if constexpr (C::SV == SV_TRI) {
                    const double ai = (i >= 1) ? step_band(S, d, d.off_sl, i) : 0.0;
                    const double ci = step_band(S, d, d.off_su, i);
                    const double ac = (i >= 1) ? ai * step_band(S, d, d.off_su, i - 1) : 0.0;
                    const double dp = (i == 0) ? 1.0 : 1.0 - ac / dprev;
                    const double m = 1.0 / dp;
                    dprev = dp;
                    l = ai * m;
                    h = ci * m;
#pragma unroll
                    for (int k = 0; k < C::NB; ++k) w[k] *= m;
                } else if constexpr (C::SV == SV_LOWER) {
                    l = (i >= 1) ? step_band(S, d, d.off_sl, i) : 0.0;
                } else if constexpr (C::SV == SV_UPPER) {
                    h = step_band(S, d, d.off_su, i);
                }
            } else if constexpr (C::SV == SV_TRI) {
                dprev = 1.0;
            }
            const int tt = (int)(i / R), jj = (int)(i % R);
            auto put = [&](int p, double v) { tb[((((size_t)s * C::NPL + p) * U + (jj >> 1)) * T + tt) * 2 + (jj & 1)] = v; };
#pragma unroll
            for (int k = 0; k < C::NB; ++k) put(k, w[k]);
            if constexpr (C::FWD) put(C::P_L, l);
            if constexpr (C::BWD) put(C::P_H, h);
        }
        __syncthreads();
    }
}

// Rows [r0, r0 + R) of one system: loaded (zero outside [0, lim) and the
// keep-window) or stored (only inside [0, lim) and the window).
template <int R>
__device__ __forceinline__ void ks_load(const double* base, int64_t r0, int64_t lim, int64_t z0, int64_t z1,
                                        bool vec, double (&x)[R])
{
    const int64_t hi = lim < z1 ? lim : z1;
#pragma unroll
    for (int u = 0; u < R / 2; ++u) {
        const int64_t r = r0 + 2 * u;
        if (vec && r >= z0 && r + 1 < hi) {
            const double2 v = __ldcs(reinterpret_cast<const double2*>(base + r));
            x[2 * u] = v.x;
            x[2 * u + 1] = v.y;
        } else {
            x[2 * u] = (r >= z0 && r < hi) ? __ldcs(base + r) : 0.0;
            x[2 * u + 1] = (r + 1 >= z0 && r + 1 < hi) ? __ldcs(base + r + 1) : 0.0;
        }
    }
}

template <int R>
__device__ __forceinline__ void ks_store(double* base, int64_t r0, int64_t lim, int64_t z0, int64_t z1, bool vec,
                                         const double (&x)[R])
{
    const int64_t hi = lim < z1 ? lim : z1;
#pragma unroll
    for (int u = 0; u < R / 2; ++u) {
        const int64_t r = r0 + 2 * u;
        if (vec && r >= z0 && r + 1 < hi) {
            __stcs(reinterpret_cast<double2*>(base + r), make_double2(x[2 * u], x[2 * u + 1]));
        } else {
            if (r >= z0 && r < hi) __stcs(base + r, x[2 * u]);
            if (r + 1 >= z0 && r + 1 < hi) __stcs(base + r + 1, x[2 * u + 1]);
        }
    }
}

template <class C>
__global__ void __launch_bounds__(C::kMaxThreads) jw_steps_kernel(const __grid_constant__ JwSteps S, const JwIO io, const int W)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int R = C::R, U = C::U, KL = C::KL, KU = C::KU;
    using O = VOps<double>;
    const int T = 32 * W;
    const int G = blockDim.x / T;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = warp / W, wg = warp - grp * W;
    double2* table = reinterpret_cast<double2*>(smem_raw);
    double* scratch_all = reinterpret_cast<double*>(smem_raw + ks_table_bytes<C>(S.K, T));

    ks_prologue<C>(S, table, scratch_all, T);

    GroupCtx g;
    g.lane = lane;
    g.wg = wg;
    g.W = W;
    g.nthr = T;
    g.bar_id = 1 + grp;
    g.seq = 0;
    g.scratch = scratch_all + (size_t)grp * W * kScratchPerWarp;
    const int t = wg * 32 + lane;
    const int64_t r0 = (int64_t)t * R;
    const double2* tb = table + t;

    const bool vec = ((reinterpret_cast<uintptr_t>(io.in) | reinterpret_cast<uintptr_t>(io.out)) & 15) == 0 &&
                     ((io.in_off | io.in_stride | io.out_off | io.out_stride) & 1) == 0;
    const int64_t step = (int64_t)gridDim.x * G;
    int64_t sys = (int64_t)blockIdx.x * G + grp;
    if (sys >= io.nsys) return;
    double x[R], nx[R];
    ks_load<R>(io.in + io.in_off + sys * io.in_stride, r0, S.M_in, io.iz0, io.iz1, vec, x);
    for (; sys < io.nsys; sys += step) {
        const bool more = sys + step < io.nsys;
        if (more) ks_load<R>(io.in + io.in_off + (sys + step) * io.in_stride, r0, S.M_in, io.iz0, io.iz1, vec, nx);
        for (int s = 0; s < S.K; ++s) {
            const double2* ts = tb + (size_t)s * C::NPL * U * T;
            auto coef = [&](int p, int u) -> double2 { return ts[(p * U + u) * T]; };
            if constexpr (C::MV) {
                double prev = 0.0, next = 0.0;
                if constexpr (KL + KU > 0) group_neighbours<double>(g, x[0], x[R - 1], prev, next);
                double y[R];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const double2 wd = coef(KL, u);
                    y[2 * u] = wd.x * x[2 * u];
                    y[2 * u + 1] = wd.y * x[2 * u + 1];
                    if constexpr (KU > 0) {
                        const double2 wu = coef(KL + 1, u);
                        y[2 * u] = O::fma(wu.x, x[2 * u + 1], y[2 * u]);
                        y[2 * u + 1] = O::fma(wu.y, (2 * u + 2 < R) ? x[2 * u + 2] : next, y[2 * u + 1]);
                    }
                    if constexpr (KL > 0) {
                        const double2 wl = coef(KL - 1, u);
                        y[2 * u] = O::fma(wl.x, (u > 0) ? x[2 * u - 1] : prev, y[2 * u]);
                        y[2 * u + 1] = O::fma(wl.y, x[2 * u], y[2 * u + 1]);
                    }
                }
#pragma unroll
                for (int j = 0; j < R; ++j) x[j] = y[j];
            }
            if constexpr (C::SV != SV_NONE) {
                auto lget = [&](int j) -> double {
                    const double2 c = coef(C::P_L, j >> 1);
                    return (j & 1) ? c.y : c.x;
                };
                auto hget = [&](int j) -> double {
                    const double2 c = coef(C::P_H, j >> 1);
                    return (j & 1) ? c.y : c.x;
                };
                chunk_solve<R, C::SV, double, double>(g, lget, hget, x);
                if (t == 0) x[0] = S.scaleC * x[0];
            }
        }
        ks_store<R>(io.out + io.out_off + sys * io.out_stride, r0, S.M_out, io.oz0, io.oz1, vec, x);
        if (more) {
#pragma unroll
            for (int j = 0; j < R; ++j) x[j] = nx[j];
        }
    }
}

}  // namespace pfb
