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

template <int R, int KL, int KU, int SV, bool DDMEM, bool TBL = false>
struct DdCfg {
    static constexpr int kR = R, kKL = KL, kKU = KU, kSV = SV;
    static constexpr bool kDdMem = DDMEM;
    static constexpr int NB = KL + KU + 1;
    static constexpr int SEG = 32 * R + KL + KU;
    static constexpr bool kFwd = (SV == SV_LOWER || SV == SV_TRI);
    static constexpr bool kBwd = (SV == SV_UPPER || SV == SV_TRI);
    // Table form (jw_dd_tbl_kernel): the step's coefficients, their chunk
    // products and the scans' multipliers in shared memory, built once per
    // CTA.  Planes of one double-double per (row of a chunk, thread): NB
    // weights, then -l and its prefix products over the chunk (forward), then
    // -h and its suffix products (backward).
    static constexpr bool kTbl = TBL;
    static constexpr int P_NL = NB, P_PL = NB + 1;
    static constexpr int P_NH = NB + (kFwd ? 2 : 0), P_PH = P_NH + 1;
    static constexpr int NP = NB + (kFwd ? 2 : 0) + (kBwd ? 2 : 0);
    static constexpr int kMul = 7;  // ScanMul<dd>: 5 levels, Ae, Aw
};

template <class C>
__host__ __device__ constexpr size_t dd_smem_per_warp()
{
    return 2 * (size_t)C::SEG * sizeof(dd);
}

// Table form: table (NP planes x R rows x 32 W threads) and the scan
// multipliers (2 directions x kMul x 32 W threads), double-doubles, after the
// staging buffers and the scan scratch.
template <class C>
__host__ __device__ constexpr size_t dd_tbl_bytes(int W)
{
    return C::kTbl ? ((size_t)C::NP * C::kR + 2 * C::kMul) * 32 * W * sizeof(dd) : 0;
}

template <class C>
__host__ size_t dd_smem_bytes(int W, int G)
{
    return (size_t)G * W * dd_smem_per_warp<C>() + (size_t)G * W * kScratchPerWarp * sizeof(double) +
           dd_tbl_bytes<C>(W);
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
            const dd na = dd_fma(a, pa, b * pc), nb = dd_fma(a, pb, b * pd);
            const dd nc = dd_fma(c, pa, d * pc), nd = dd_fma(c, pb, d * pd);
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
            const dd na = dd_fma(oa, wa, ob * wc), nb = dd_fma(oa, wb, ob * wd);
            const dd nc = dd_fma(oc, wa, od * wc), nd = dd_fma(oc, wb, od * wd);
            wa = na; wb = nb; wc = nc; wd = nd;
            renorm2x2_dd(wa, wb, wc, wd);
        }
        group_bar(g.bar_id, g.nthr);
    }
    a = dd_fma(ea, wa, eb * wc);
    b = dd_fma(ea, wb, eb * wd);
    c = dd_fma(ec, wa, ed * wc);
    d = dd_fma(ec, wb, ed * wd);
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


// ---- Table form of the double-double step.
//
// jw_dd_kernel keeps each thread's coefficients in registers, which holds it
// at 4 or 8 rows per thread, and recomputes per system the chunk products of
// the solve bands and the scans' multipliers.  None of them depend on the
// right-hand side: here group 0 builds them once per CTA into shared memory
// (the coefficients row by row, so no thread holds a chunk's worth), and every
// system then costs per row one double-double multiply-add for the local
// recurrence and one for the coupling, in each direction, plus the matvec.
// With 8 or 16 rows per thread the scans are amortised over more rows, and
// systems of up to 512 rows run on one warp, without cross-warp barriers.

// The table, built by all NT threads of the CTA: thread tid takes rows
// [tid Rp, tid Rp + Rp) of the group's T R rows (their pivots from a Moebius
// scan over the CTA, as dd_prologue does over a group), then group 0 (tid <
// T: one thread per chunk) forms the chunk products and the scans'
// multipliers.  Same values as dd_prologue and chunk_solve compute per
// system, up to the association of the pivot products.
template <class C>
__device__ __noinline__ void dd_tbl_prologue(const JwOperator& op, dd* tab, dd* mul, double* scratch_all, int T,
                                             int NT)
{
    constexpr int R = C::kR, KL = C::kKL, KU = C::kKU, NB = C::NB;
    const int64_t M = op.M;
    const int tid = threadIdx.x;
    auto bnd = [&](int64_t off, int64_t i) { return band_dd<C::kDdMem>(op.bands, off, band_pos(op, i)); };
    auto at = [&](int p, int64_t i) -> dd& { return tab[((size_t)p * R + (i % R)) * T + (i / R)]; };
    GroupCtx gc;
    gc.lane = tid & 31;
    gc.wg = tid >> 5;
    gc.W = NT >> 5;
    gc.nthr = NT;
    gc.bar_id = 1;
    gc.seq = 0;
    gc.scratch = scratch_all;
    const int rows = T * R;
    const int Rp = (rows + NT - 1) / NT;
    const int64_t s = (int64_t)tid * Rp;
    dd dprev(1.0);
    if constexpr (C::kSV == SV_TRI) {
        dd a(1.0), b(0.0), c(0.0), d(1.0);
        for (int j = 0; j < Rp; ++j) {
            const int64_t i = s + j;
            dd ac(0.0);
            if (i >= 1 && i < M) ac = bnd(op.off_sl, i) * ((i - 1 < M - 1) ? bnd(op.off_su, i - 1) : dd(0.0));
            const dd na = a - ac * c, nb = b - ac * d;
            c = a;
            d = b;
            a = na;
            b = nb;
            renorm2x2_dd(a, b, c, d);
        }
        group_matrix_scan_dd(gc, a, b, c, d);
        dprev = (s == 0) ? dd(1.0) : a / c;
    }
#pragma unroll 1
    for (int j = 0; j < Rp; ++j) {
        const int64_t i = s + j;
        if (i >= rows) break;
        dd w[NB];
#pragma unroll
        for (int k = 0; k < NB; ++k) w[k] = dd(0.0);
        dd nl(0.0), nh(0.0);
        if (i < M) {
            dd vl(0.0), vd(1.0), vu(0.0);
            if (op.mvj != MVJ_NONE) vd = bnd(op.off_md, i);
            if (op.mvj == MVJ_UPPER && i + 1 < M) vu = bnd(op.off_mo, i);
            if (op.mvj == MVJ_LOWER && i >= 1) vl = bnd(op.off_mo, i);
            if (op.dgbmv == nullptr) {
                if constexpr (KL >= 1) w[KL - 1] = vl;
                w[KL] = vd;
                if constexpr (KU >= 1) w[KL + 1] = vu;
            } else {
                const int kla = op.dg_lda - 1 - op.dg_ku;
                for (int pv = -1; pv <= 1; ++pv) {
                    const dd vp = (pv < 0) ? vl : (pv == 0 ? vd : vu);
                    const int64_t q = i + pv;
                    if (dd_is_zero(vp) || q < 0 || q >= M) continue;
                    for (int kk = -kla; kk <= op.dg_ku; ++kk) {
                        const int64_t cc = q + kk;
                        if (cc < 0 || cc >= M) continue;
                        const dd av = band_dd<C::kDdMem>(op.dgbmv, op.dg_off, (int64_t)(op.dg_ku - kk) * M + cc);
                        const int k = (int)(cc - i);
#pragma unroll
                        for (int qq = 0; qq < NB; ++qq)
                            if (qq - KL == k) w[qq] = dd_fma(vp, av, w[qq]);
                    }
                }
            }
            if constexpr (C::kSV == SV_TRI) {
                const dd ai = (i >= 1) ? bnd(op.off_sl, i) : dd(0.0);
                const dd ci = (i < M - 1) ? bnd(op.off_su, i) : dd(0.0);
                const dd ac = (i >= 1) ? ai * ((i - 1 < M - 1) ? bnd(op.off_su, i - 1) : dd(0.0)) : dd(0.0);
                const dd dp = (i == 0) ? dd(1.0) : dd(1.0) - ac / dprev;
                const dd dinv = dd(1.0) / dp;
                dprev = dp;
                nl = -(ai * dinv);
                nh = -(ci * dinv);
#pragma unroll
                for (int k = 0; k < NB; ++k) w[k] = w[k] * dinv;
            } else if constexpr (C::kSV == SV_LOWER) {
                nl = (i >= 1) ? -bnd(op.off_sl, i) : dd(0.0);
            } else if constexpr (C::kSV == SV_UPPER) {
                nh = (i < M - 1) ? -bnd(op.off_su, i) : dd(0.0);
            }
        }
#pragma unroll
        for (int k = 0; k < NB; ++k) at(k, i) = w[k];
        if constexpr (C::kFwd) at(C::P_NL, i) = nl;
        if constexpr (C::kBwd) at(C::P_NH, i) = nh;
    }
    __syncthreads();
    if (tid >= T) return;
    // group 0, thread t = tid: its chunk's products and the scans' multipliers
    GroupCtx g = gc;
    g.W = T >> 5;
    g.nthr = T;
    const int t = tid;
    auto ch = [&](int p, int j) -> dd& { return tab[((size_t)p * R + j) * T + t]; };
    if constexpr (C::kFwd) {
        dd p(1.0);
#pragma unroll 1
        for (int j = 0; j < R; ++j) {
            p = ch(C::P_NL, j) * p;
            ch(C::P_PL, j) = p;
        }
        const ScanMul<dd> m = scan_multipliers<dd, true>(g, p);
#pragma unroll
        for (int k = 0; k < 5; ++k) mul[k * T + t] = m.lev[k];
        mul[5 * T + t] = m.Ae;
        mul[6 * T + t] = m.Aw;
    }
    if constexpr (C::kBwd) {
        dd p(1.0);
#pragma unroll 1
        for (int j = R - 1; j >= 0; --j) {
            p = ch(C::P_NH, j) * p;
            ch(C::P_PH, j) = p;
        }
        const ScanMul<dd> m = scan_multipliers<dd, false>(g, p);
#pragma unroll
        for (int k = 0; k < 5; ++k) mul[(C::kMul + k) * T + t] = m.lev[k];
        mul[(C::kMul + 5) * T + t] = m.Ae;
        mul[(C::kMul + 6) * T + t] = m.Aw;
    }
}

template <class C>
__global__ void __launch_bounds__(256, C::kR <= 8 ? 2 : 1) jw_dd_tbl_kernel(const JwOperator op, const JwIO io, const int W)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int R = C::kR, KL = C::kKL, KU = C::kKU;
    const int warp = threadIdx.x >> 5;
    const int G = blockDim.x / (32 * W);
    const int grp = warp / W;
    const int T = 32 * W;
    GroupCtx g;
    g.lane = threadIdx.x & 31;
    g.wg = warp - grp * W;
    g.W = W;
    g.nthr = T;
    g.bar_id = 1 + grp;
    g.seq = 0;
    constexpr size_t per_warp = dd_smem_per_warp<C>();
    dd* buf0 = reinterpret_cast<dd*>(smem_raw + (size_t)warp * per_warp);
    dd* buf1 = buf0 + C::SEG;
    double* scratch_all = reinterpret_cast<double*>(smem_raw + (size_t)G * W * per_warp);
    g.scratch = scratch_all + (size_t)grp * W * kScratchPerWarp;
    dd* tab = reinterpret_cast<dd*>(scratch_all + (size_t)G * W * kScratchPerWarp);
    dd* mul = tab + (size_t)C::NP * R * T;
    const int t = g.wg * 32 + g.lane;  // thread of the group: its chunk
    const int64_t r0 = (int64_t)g.wg * 32 * R;
    const int64_t s = (int64_t)t * R;
    const int64_t sys0 = (int64_t)blockIdx.x * G + grp;
    const int64_t step = (int64_t)gridDim.x * G;
    // the first system's copy is in flight while the CTA builds the table
    if (sys0 < io.nsys) dd_issue_load<C>(io, sys0, r0, g.lane, buf0);
    cp_async_commit();
    dd_tbl_prologue<C>(op, tab, mul, scratch_all, T, (int)blockDim.x);
    __syncthreads();
    g.seq = 0;
    auto co = [&](int p, int j) -> dd { return tab[((size_t)p * R + j) * T + t]; };
    ScanMul<dd> mf, mb;
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
        dd x[R + KL + KU];
#pragma unroll
        for (int j = 0; j < R + KL + KU; ++j) {
            const int q = g.lane * R + j - KL;
            int slot;
            if (q < 0) slot = 32 * R + (q + KL);
            else if (q >= 32 * R) slot = 32 * R + KL + (q - 32 * R);
            else slot = swz<R, true>(q);
            x[j] = cur[slot];
        }
#pragma unroll
        for (int j = 0; j < R; ++j) {
            dd acc = co(0, j) * x[j];
#pragma unroll
            for (int k = 1; k < C::NB; ++k) acc = dd_fma(co(k, j), x[j + k], acc);
            x[j] = acc;
        }
        if constexpr (C::kFwd) {
#pragma unroll
            for (int j = 1; j < R; ++j) x[j] = dd_fma(co(C::P_NL, j), x[j - 1], x[j]);
#pragma unroll
            for (int k = 0; k < 5; ++k) mf.lev[k] = mul[k * T + t];
            mf.Ae = mul[5 * T + t];
            mf.Aw = mul[6 * T + t];
            const dd pin = group_affine_scan_pre<dd, dd, true>(g, mf, x[R - 1]);
#pragma unroll
            for (int j = 0; j < R; ++j) x[j] = dd_fma(co(C::P_PL, j), pin, x[j]);
        }
        if constexpr (C::kBwd) {
#pragma unroll
            for (int j = R - 2; j >= 0; --j) x[j] = dd_fma(co(C::P_NH, j), x[j + 1], x[j]);
#pragma unroll
            for (int k = 0; k < 5; ++k) mb.lev[k] = mul[(C::kMul + k) * T + t];
            mb.Ae = mul[(C::kMul + 5) * T + t];
            mb.Aw = mul[(C::kMul + 6) * T + t];
            const dd q = group_affine_scan_pre<dd, dd, false>(g, mb, x[0]);
#pragma unroll
            for (int j = 0; j < R; ++j) x[j] = dd_fma(co(C::P_PH, j), q, x[j]);
        }
        if constexpr (C::kSV != SV_NONE) {
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
