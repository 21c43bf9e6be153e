// dd_kernel.cuh -- the JW step in double-double arithmetic (quad emulation).
//
// Same operator and partition method as jw_kernel.cuh, with every value and
// coefficient an unevaluated double-double (dd.cuh):
//   x = M^{-1} * (V * A * b),  x[0] *= scaleC when a solve runs
// for real right-hand sides stored either as double-double pairs {hi, lo}
// (PfSolve's quadDoubleDoublePrecision, 16 B per value) or as FP64
// (quadDoubleDoublePrecisionDoubleMemory; results rounded to FP64).
// The tridiagonal pivots come from a double-double Moebius scan, so no
// thread walks all N rows; all arithmetic of the step is FP64-pipe work
// (~20 FP64 operations per double-double multiply-add).
#pragma once
#include "jw_kernel.cuh"

namespace pfb {

template <int R, int KL, int KU, int SV, bool DDMEM>
struct DdCfg {
    static constexpr int kR = R, kKL = KL, kKU = KU, kSV = SV;
    static constexpr bool kDdMem = DDMEM;
    static constexpr int NB = KL + KU + 1;
    static constexpr int SEG = 32 * R + KL + KU;
    static constexpr bool kFwd = (SV == SV_LOWER || SV == SV_TRI);
    static constexpr bool kBwd = (SV == SV_UPPER || SV == SV_TRI);
};

template <class C>
__host__ __device__ constexpr size_t dd_smem_per_warp()
{
    return 2 * (size_t)C::SEG * sizeof(dd);
}

template <class C>
__host__ size_t dd_smem_bytes(int W, int G)
{
    return (size_t)G * W * dd_smem_per_warp<C>() + (size_t)G * W * kScratchPerWarp * sizeof(double);
}

// Band value of logical row i as double-double (dd storage: pairs).
template <bool DDMEM>
__device__ __forceinline__ dd band_dd(const double* base, int64_t off, int64_t pos)
{
    if constexpr (DDMEM) return dd(__ldg(base + 2 * (off + pos)), __ldg(base + 2 * (off + pos) + 1));
    else return dd(__ldg(base + off + pos));
}

__device__ __forceinline__ void renorm2x2_dd(dd& a, dd& b, dd& c, dd& d)
{
    double m = fmax(fmax(fabs(a.hi), fabs(b.hi)), fmax(fabs(c.hi), fabs(d.hi)));
    if (m > 0.0 && isfinite(m)) {
        const int e = ilogb(m);
        a = dd(scalbn(a.hi, -e), scalbn(a.lo, -e));
        b = dd(scalbn(b.hi, -e), scalbn(b.lo, -e));
        c = dd(scalbn(c.hi, -e), scalbn(c.lo, -e));
        d = dd(scalbn(d.hi, -e), scalbn(d.lo, -e));
    }
}

// Exclusive scan of 2x2 double-double matrix products (row order).
__device__ __forceinline__ void group_matrix_scan_dd(GroupCtx& g, dd& a, dd& b, dd& c, dd& d)
{
    using O = VOps<dd>;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
        const dd pa = O::shfl_up(a, s), pb = O::shfl_up(b, s), pc = O::shfl_up(c, s), pd = O::shfl_up(d, s);
        if (g.lane >= s) {
            const dd na = a * pa + b * pc, nb = a * pb + b * pd;
            const dd nc = c * pa + d * pc, nd = c * pb + d * pd;
            a = na; b = nb; c = nc; d = nd;
            renorm2x2_dd(a, b, c, d);
        }
    }
    dd ea = O::shfl_up(a, 1), eb = O::shfl_up(b, 1), ec = O::shfl_up(c, 1), ed = O::shfl_up(d, 1);
    if (g.lane == 0) { ea = dd(1.0); eb = dd(0.0); ec = dd(0.0); ed = dd(1.0); }
    dd wa(1.0), wb(0.0), wc(0.0), wd(1.0);
    if (g.W > 1) {
        // warp aggregates: 8 doubles at [16, 24) of each warp's scratch
        double* my = g.warp_area(g.wg) + 16;
        if (g.lane == 31) {
            store_v<dd>(my, a); store_v<dd>(my + 2, b); store_v<dd>(my + 4, c); store_v<dd>(my + 6, d);
        }
        __syncwarp();
        group_bar(g.bar_id, g.nthr);
        for (int w = 0; w < g.wg; ++w) {
            const double* o = g.warp_area(w) + 16;
            const dd oa = load_v<dd>(o), ob = load_v<dd>(o + 2), oc = load_v<dd>(o + 4), od = load_v<dd>(o + 6);
            const dd na = oa * wa + ob * wc, nb = oa * wb + ob * wd;
            const dd nc = oc * wa + od * wc, nd = oc * wb + od * wd;
            wa = na; wb = nb; wc = nc; wd = nd;
            renorm2x2_dd(wa, wb, wc, wd);
        }
        group_bar(g.bar_id, g.nthr);
    }
    a = ea * wa + eb * wc;
    b = ea * wb + eb * wd;
    c = ec * wa + ed * wc;
    d = ec * wb + ed * wd;
}

template <class C>
struct DdCoef {
    dd w[C::NB][C::kR];
    dd l[C::kFwd ? C::kR : 1];
    dd h[C::kBwd ? C::kR : 1];
};

template <class C>
__device__ __forceinline__ void dd_prologue(const JwOperator& op, GroupCtx& g, int64_t s, DdCoef<C>& cf)
{
    constexpr int R = C::kR, KL = C::kKL, KU = C::kKU;
    const int64_t M = op.M;
    auto bnd = [&](int64_t off, int64_t i) { return band_dd<C::kDdMem>(op.bands, off, band_pos(op, i)); };
#pragma unroll
    for (int j = 0; j < R; ++j) {
#pragma unroll
        for (int k = 0; k < C::NB; ++k) cf.w[k][j] = dd(0.0);
        const int64_t i = s + j;
        if (i < M) {
            dd vl(0.0), vd(1.0), vu(0.0);
            if (op.mvj != MVJ_NONE) vd = bnd(op.off_md, i);
            if (op.mvj == MVJ_UPPER && i + 1 < M) vu = bnd(op.off_mo, i);
            if (op.mvj == MVJ_LOWER && i >= 1) vl = bnd(op.off_mo, i);
            if (op.dgbmv == nullptr) {
                if constexpr (KL >= 1) cf.w[KL - 1][j] = vl;
                cf.w[KL][j] = vd;
                if constexpr (KU >= 1) cf.w[KL + 1][j] = vu;
            } else {
                const int kla = op.dg_lda - 1 - op.dg_ku;
                for (int pv = -1; pv <= 1; ++pv) {
                    const dd vp = (pv < 0) ? vl : (pv == 0 ? vd : vu);
                    const int64_t p = i + pv;
                    if (dd_is_zero(vp) || p < 0 || p >= M) continue;
                    for (int kk = -kla; kk <= op.dg_ku; ++kk) {
                        const int64_t c = p + kk;
                        if (c < 0 || c >= M) continue;
                        const dd a = band_dd<C::kDdMem>(op.dgbmv, op.dg_off, (int64_t)(op.dg_ku - kk) * M + c);
                        const int k = (int)(c - i);
#pragma unroll
                        for (int q = 0; q < C::NB; ++q)
                            if (q - KL == k) cf.w[q][j] = dd_fma(vp, a, cf.w[q][j]);
                    }
                }
            }
        }
    }
    if constexpr (C::kSV == SV_TRI) {
        dd a(1.0), b(0.0), c(0.0), d(1.0);
        dd acs[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int64_t i = s + j;
            dd ac(0.0);
            if (i >= 1 && i < M) {
                const dd ai = bnd(op.off_sl, i);
                const dd cim1 = (i - 1 < M - 1) ? bnd(op.off_su, i - 1) : dd(0.0);
                ac = ai * cim1;
            }
            acs[j] = ac;
            const dd na = a - ac * c, nb = b - ac * d;
            c = a; d = b; a = na; b = nb;
            renorm2x2_dd(a, b, c, d);
        }
        group_matrix_scan_dd(g, a, b, c, d);
        dd dprev = (s == 0) ? dd(1.0) : a / c;
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int64_t i = s + j;
            const dd dp = (i == 0) ? dd(1.0) : dd(1.0) - acs[j] / dprev;
            const dd dinv = dd(1.0) / dp;
            dprev = dp;
            const dd ai = (i >= 1 && i < M) ? bnd(op.off_sl, i) : dd(0.0);
            const dd ci = (i < M - 1) ? bnd(op.off_su, i) : dd(0.0);
            cf.l[j] = ai * dinv;
            cf.h[j] = ci * dinv;
#pragma unroll
            for (int k = 0; k < C::NB; ++k) cf.w[k][j] = cf.w[k][j] * dinv;
        }
    } else if constexpr (C::kSV == SV_LOWER) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int64_t i = s + j;
            cf.l[j] = (i >= 1 && i < M) ? bnd(op.off_sl, i) : dd(0.0);
        }
    } else if constexpr (C::kSV == SV_UPPER) {
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const int64_t i = s + j;
            cf.h[j] = (i < M - 1) ? bnd(op.off_su, i) : dd(0.0);
        }
    }
}

template <class C>
__device__ __forceinline__ void dd_issue_load(const JwIO& io, int64_t sys, int64_t r0, int lane, dd* buf)
{
    constexpr int R = C::kR, KL = C::kKL, KU = C::kKU;
    const int64_t M = io.M;
    auto put = [&](int slot, int64_t row) {
        const bool ok = row >= 0 && row < M && row >= io.iz0 && row < io.iz1;
        double* dst = reinterpret_cast<double*>(buf + slot);
        if constexpr (C::kDdMem) {
            const double* src = io.in + 2 * (io.in_off + sys * io.in_stride + row);
            cp_async16(dst, ok ? src : io.in, ok);
        } else {
            const double* src = io.in + io.in_off + sys * io.in_stride + row;
            cp_async8(dst, ok ? src : io.in, ok);
            cp_async8(dst + 1, io.in, false);  // lo = 0
        }
    };
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int q = 32 * k + lane;
        put(swz<R, true>(q), r0 + q);
    }
    if (KL > 0 && lane < KL) put(32 * R + lane, r0 - KL + lane);
    if (KU > 0 && lane < KU) put(32 * R + KL + lane, r0 + 32 * R + lane);
}

template <class C>
__device__ __forceinline__ void dd_store(const JwIO& io, int64_t sys, int64_t r0, int lane, const dd* buf)
{
    constexpr int R = C::kR;
    const int64_t M = io.M;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int q = 32 * k + lane;
        const int64_t row = r0 + q;
        if (row >= M || row < io.oz0 || row >= io.oz1) continue;
        const dd v = buf[swz<R, true>(q)];
        if constexpr (C::kDdMem) {
            double2* p = reinterpret_cast<double2*>(io.out) + io.out_off + sys * io.out_stride + row;
            *p = make_double2(v.hi, v.lo);
        } else {
            io.out[io.out_off + sys * io.out_stride + row] = v.hi + v.lo;
        }
    }
}

template <class C>
__global__ void __launch_bounds__(256) jw_dd_kernel(const JwOperator op, const JwIO io, const int W)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using O = VOps<dd>;
    constexpr int R = C::kR, KL = C::kKL, KU = C::kKU;
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
    constexpr size_t per_warp = dd_smem_per_warp<C>();
    dd* buf0 = reinterpret_cast<dd*>(smem_raw + (size_t)warp * per_warp);
    dd* buf1 = buf0 + C::SEG;
    g.scratch = reinterpret_cast<double*>(smem_raw + (size_t)G * W * per_warp) + (size_t)grp * W * kScratchPerWarp;
    const int64_t r0 = (int64_t)g.wg * 32 * R;
    const int64_t s = r0 + (int64_t)g.lane * R;
    DdCoef<C> cf;
    dd_prologue<C>(op, g, s, cf);
    const int64_t sys0 = (int64_t)blockIdx.x * G + grp;
    const int64_t step = (int64_t)gridDim.x * G;
    if (sys0 >= io.nsys) return;
    dd_issue_load<C>(io, sys0, r0, g.lane, buf0);
    cp_async_commit();
    int it = 0;
    for (int64_t sys = sys0; sys < io.nsys; sys += step, ++it) {
        dd* cur = (it & 1) ? buf1 : buf0;
        dd* nxt = (it & 1) ? buf0 : buf1;
        if (sys + step < io.nsys) dd_issue_load<C>(io, sys + step, r0, g.lane, nxt);
        cp_async_commit();
        cp_async_wait<1>();
        __syncwarp();
        if constexpr (C::kSV == SV_NONE && (KL + KU) > 0) {
            if (g.W > 1) group_bar(g.bar_id, g.nthr);
        }
        dd be[R + KL + KU];
#pragma unroll
        for (int j = 0; j < R + KL + KU; ++j) {
            const int q = g.lane * R + j - KL;
            int slot;
            if (q < 0) slot = 32 * R + (q + KL);
            else if (q >= 32 * R) slot = 32 * R + KL + (q - 32 * R);
            else slot = swz<R, true>(q);
            be[j] = cur[slot];
        }
        dd x[R];
#pragma unroll
        for (int j = 0; j < R; ++j) {
            dd acc = cf.w[0][j] * be[j];
#pragma unroll
            for (int k = 1; k < C::NB; ++k) acc = dd_fma(cf.w[k][j], be[j + k], acc);
            x[j] = acc;
        }
        if constexpr (C::kSV != SV_NONE) {
            chunk_solve<R, C::kSV, dd, dd>(g, [&](int j) { return cf.l[j]; }, [&](int j) { return cf.h[j]; }, x);
            if (s == 0) x[0] = dd(op.scaleC) * x[0];
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < R; ++j) cur[swz<R, true>(g.lane * R + j)] = x[j];
        __syncwarp();
        dd_store<C>(io, sys, r0, g.lane, cur);
        __syncwarp();
    }
    cp_async_wait<0>();
}

}  // namespace pfb
