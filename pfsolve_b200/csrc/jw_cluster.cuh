// jw_cluster.cuh -- the JW step for long systems (N > 4096): one thread-block
// cluster per system.
//
// Same operator as the streaming kernel (x = M^{-1} V b, x[0] *= scaleC; real
// FP64 systems; PfSolve_shaderGen_JonesWorlandMV,
// PfSolve/pfSolve_CodeGen/pfSolve_KernelsLevel2/pfSolve_JonesWorland.h:38-408;
// the reference splits such systems over several kernel uploads,
// pfSolve_AppManagement/pfSolve_InitializeApp.h:1540-1583).
//
//  * A cluster of C CTAs (on C SMs) owns one system at a time; CTA c holds the
//    rows [c*S, (c+1)*S), S = 32*W*R, one group of W warps with R rows per
//    thread, and streams its slice with TMA boxes exactly as the streaming
//    kernel does (no multicast: every CTA loads and stores its own rows).
//  * The matvec halo rows at slice ends are read from the neighbour CTA's
//    shared memory (mapa + ld.shared::cluster) after a cluster barrier.
//  * The scans run in two levels: the group scan gives every thread the affine
//    map from the value entering its CTA to the value entering its chunk; the
//    CTAs' total maps are published in shared memory, a cluster barrier later
//    each CTA composes those of the CTAs before it (forward) or after it
//    (backward).  The tridiagonal pivots' Moebius scan is composed the same
//    way in the prologue.
//  * Cluster barriers are mbarrier-based (remote arrivals, a bounded wait),
//    and a CTA publishes whether the TMA load of a system completed before
//    the barrier that precedes the system's first shared-memory exchange (the
//    last barrier of the previous system), so all CTAs of the cluster stop
//    together when one load did not complete, and one barrier per system
//    serves both the previous system's scan and the next one's halo.  A
//    barrier whose peers never arrive ends with a status bit instead of a
//    hang.
#pragma once
#include "jw_stream.cuh"

namespace pfb {

template <int R_, int W_, int C_, int KL_, int KU_, int SV_>
struct ClCfg {
    using B = StCfg<R_, W_, KL_, KU_, SV_, LAY_REAL, LAY_REAL, false, PREC_F64, 0, 0>;  // slice layout and table planes
    static constexpr int C = C_;
    static constexpr int R = R_, W = W_, T = 32 * W_, S = T * R_;
    static constexpr int KL = KL_, KU = KU_, SV = SV_;
    // per-parity exchange slots, in doubles: forward map (A, B), backward map,
    // wait status, Moebius aggregate (4)
    static constexpr int XF = 0, XB = 2, XOK = 4, XM = 8, XN = 12;
    static constexpr size_t XCHG = 2 * XN * sizeof(double);
};

template <class C>
__host__ __device__ constexpr size_t cl_smem_bytes()
{
    return C::B::TBL + (size_t)C::W * kScratchPerWarp * sizeof(double) + C::XCHG + 4 * sizeof(uint64_t) + 1024 +
           2 * C::B::BUF;
}

__device__ __forceinline__ uint32_t cluster_ctarank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_id_x()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;\n" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t num_clusters_x()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;\n" : "=r"(r));
    return r;
}
// Every thread of every CTA of the cluster; release/acquire orders shared
// memory writes before the barrier with reads after it, cluster-wide.
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ uint32_t mapa_rank(uint32_t local, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(local), "r"(rank));
    return r;
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t remote_bar)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(remote_bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait_cluster(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Barrier over the CTAs of the cluster, built on one mbarrier per CTA (C
// arrivals per phase): after the CTA's own threads meet, the CTA arrives with
// release semantics on every CTA's mbarrier, and thread 0 waits -- for about
// two seconds at most -- for the arrivals of all CTAs.  Returns false when
// that wait ran out; the caller then stops.  A CTA may arrive for the next
// barrier before a slower peer's current phase completes; that arrival only
// lands after every CTA has arrived for the current one, so each phase still
// completes only once all CTAs reached the barrier, and no phase is skipped.
template <int C>
__device__ __forceinline__ bool cl_barrier(uint32_t cbar, uint32_t& phase, volatile int* flag, int nthr)
{
    group_bar(1, nthr);
    // lanes 0..C-1 of warp 0 arrive on one CTA each; the release covers the
    // CTA's writes ordered before the bar.sync above
    if (threadIdx.x < C) mbar_arrive_remote(mapa_rank(cbar, threadIdx.x));
    if (threadIdx.x == 0) {
        bool ok = mbar_try_wait_cluster(cbar, phase);
        if (!ok) {
            const long long t0 = clock64();
            while (!(ok = mbar_try_wait_cluster(cbar, phase)))
                if (clock64() - t0 > 4000000000LL) break;
        }
        *flag = ok ? 1 : 0;
    }
    group_bar(1, nthr);
    phase ^= 1u;
    return *flag != 0;
}

// Status bits of a cluster barrier that ran out, by barrier (kStatusWaitTimeout
// is also set).
constexpr unsigned kStatusClusterBarrier = 1u << 8;

__device__ __forceinline__ double ld_cluster_f64(uint32_t addr)
{
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];\n" : "=d"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ double2 ld_cluster_v2(uint32_t addr)
{
    double2 v;
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "r"(addr) : "memory");
    return v;
}

// Scan of affine maps y = B + A x over the group (row order forward, reverse
// order backward).  Returns, for this thread, the map (Ain, Bin) from the
// value entering the group to the value entering this thread's chunk, and the
// group's total map (Atot, Btot) (identical in every thread).
template <bool FORWARD>
__device__ __forceinline__ void group_affine_scan_map(GroupCtx& g, double A, double B, double& Ain, double& Bin,
                                                      double& Atot, double& Btot)
{
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double Ap = FORWARD ? __shfl_up_sync(FULL, A, d) : __shfl_down_sync(FULL, A, d);
        const double Bp = FORWARD ? __shfl_up_sync(FULL, B, d) : __shfl_down_sync(FULL, B, d);
        const bool take = FORWARD ? (g.lane >= d) : (g.lane + d < 32);
        if (take) {
            B = __fma_rn(A, Bp, B);
            A = A * Ap;
        }
    }
    double Ae = FORWARD ? __shfl_up_sync(FULL, A, 1) : __shfl_down_sync(FULL, A, 1);
    double Be = FORWARD ? __shfl_up_sync(FULL, B, 1) : __shfl_down_sync(FULL, B, 1);
    const int last = FORWARD ? 31 : 0;
    if (g.lane == (FORWARD ? 0 : 31)) {
        Ae = 1.0;
        Be = 0.0;
    }
    const double Aw_agg = __shfl_sync(FULL, A, last), Bw_agg = __shfl_sync(FULL, B, last);
    double Aw = 1.0, Bw = 0.0;  // group input -> this warp's input
    double At = Aw_agg, Bt = Bw_agg;
    if (g.W > 1) {
        const int slot = (FORWARD ? 0 : 8) + 4 * (g.seq & 1);
        if (g.lane == last) {
            double* my = g.warp_area(g.wg) + slot;
            my[0] = A;
            my[2] = B;
        }
        __syncwarp();
        group_bar(g.bar_id, g.nthr);
        At = 1.0;
        Bt = 0.0;
        for (int k = 0; k < g.W; ++k) {
            const int w = FORWARD ? k : g.W - 1 - k;
            const double* o = g.warp_area(w) + slot;
            if (w == g.wg) {
                Aw = At;
                Bw = Bt;
            }
            Bt = __fma_rn(o[0], Bt, o[2]);
            At = o[0] * At;
        }
        g.seq++;
    }
    Ain = Ae * Aw;
    Bin = __fma_rn(Ae, Bw, Be);
    Atot = At;
    Btot = Bt;
}

// ---- Coefficient table of this CTA's slice (rows crank*S + [0, S)), built by
// all its threads; the Moebius pivots are scanned across the cluster.
template <class C>
__device__ bool cl_prologue(const JwOperator& op, double* table, double* scratch, double* xchg, uint32_t crank,
                            uint32_t cbar, uint32_t& cphase, volatile int* cflag)
{
    using BC = typename C::B;
    constexpr int R = C::R, U = BC::U, NB = BC::NB, S = C::S;
    const int64_t M = op.M;
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int Rp = (S + nthr - 1) / nthr;
    const int64_t s0 = (int64_t)crank * S;  // first row of the slice
    const int64_t s = s0 + (int64_t)tid * Rp;
    GroupCtx g;
    g.lane = tid & 31;
    g.wg = tid >> 5;
    g.W = nthr >> 5;
    g.nthr = nthr;
    g.bar_id = 1;
    g.seq = 0;
    g.scratch = scratch;
    double dprev = 1.0;
    if constexpr (C::SV == SV_TRI) {
        double a = 1, b = 0, c = 0, d = 1;
        for (int j = 0; j < Rp; ++j) {
            const int64_t i = s + j;
            double ac = 0.0;
            if (i >= 1 && i < M && i < s0 + S) ac = band(op, op.off_sl, i) * band(op, op.off_su, i - 1);
            const double na = a - ac * c, nb = b - ac * d;
            c = a;
            d = b;
            a = na;
            b = nb;
            renorm2x2(a, b, c, d);
        }
        const double pa = a, pb = b, pc = c, pd = d;  // this thread's product
        group_matrix_scan(g, a, b, c, d);            // product of the CTA's preceding chunks
        // CTA aggregate = own * preceding (last thread), published per CTA
        if (tid == nthr - 1) {
            double na = pa * a + pb * c, nb = pa * b + pb * d, nc = pc * a + pd * c, nd = pc * b + pd * d;
            renorm2x2(na, nb, nc, nd);
            xchg[C::XM + 0] = na;
            xchg[C::XM + 1] = nb;
            xchg[C::XM + 2] = nc;
            xchg[C::XM + 3] = nd;
        }
        if (!cl_barrier<C::C>(cbar, cphase, cflag, nthr)) return false;
        // preceding CTAs: Q = agg[c-1] * ... * agg[0]
        double qa = 1, qb = 0, qc = 0, qd = 1;
        const uint32_t xm = smem_u32(xchg + C::XM);
        for (uint32_t r = 0; r < crank; ++r) {
            const uint32_t ra = mapa_rank(xm, r);
            const double oa = ld_cluster_f64(ra), ob = ld_cluster_f64(ra + 8), oc = ld_cluster_f64(ra + 16),
                         od = ld_cluster_f64(ra + 24);
            double na = oa * qa + ob * qc, nb = oa * qb + ob * qd, nc = oc * qa + od * qc, nd = oc * qb + od * qd;
            renorm2x2(na, nb, nc, nd);
            qa = na;
            qb = nb;
            qc = nc;
            qd = nd;
        }
        // full prefix = (CTA prefix) * Q; incoming vector = prefix * (1, 0)^T
        const double fa = a * qa + b * qc, fc = c * qa + d * qc;
        dprev = (s == 0) ? 1.0 : fa / fc;
    }
    for (int j = 0; j < Rp; ++j) {
        const int64_t li = (int64_t)tid * Rp + j;  // row within the slice
        if (li >= S) break;
        const int64_t i = s0 + li;
        double w[NB];
        double nl = 0.0, nh = 0.0;
        if (i < M) {
            jw_row_weights<C::KL, NB>(op, i, w);
            double m = 1.0;
            if constexpr (C::SV == SV_TRI) {
                const double ai = (i >= 1) ? band(op, op.off_sl, i) : 0.0;
                const double ci = (i < M - 1) ? band(op, op.off_su, i) : 0.0;
                const double ac = (i >= 1) ? ai * band(op, op.off_su, i - 1) : 0.0;
                const double dp = (i == 0) ? 1.0 : 1.0 - ac / dprev;
                m = 1.0 / dp;
                dprev = dp;
                nl = -(ai * m);
                nh = -(ci * m);
            } else if constexpr (C::SV == SV_LOWER) {
                nl = (i >= 1) ? -band(op, op.off_sl, i) : 0.0;
            } else if constexpr (C::SV == SV_UPPER) {
                nh = (i < M - 1) ? -band(op, op.off_su, i) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < NB; ++k) w[k] *= m;
        } else {
#pragma unroll
            for (int k = 0; k < NB; ++k) w[k] = 0.0;
        }
        const int tt = (int)(li / R), jj = (int)(li % R);
        auto put = [&](int p, double v) { table[(((size_t)p * U + (jj >> 1)) * BC::TP + tt) * 2 + (jj & 1)] = v; };
#pragma unroll
        for (int k = 0; k < NB; ++k) put(k, w[k]);
        if constexpr (BC::FWD) put(BC::P_NL, nl);
        if constexpr (BC::BWD) put(BC::P_NH, nh);
    }
    return true;
}

template <class C>
__global__ void __launch_bounds__(C::T) jw_cluster_kernel(const __grid_constant__ CUtensorMap tm_in,
                                                         const __grid_constant__ CUtensorMap tm_out,
                                                         const JwOperator op, const JwIO io)
{
    using BC = typename C::B;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int R = C::R, W = C::W, T = C::T, U = BC::U, KL = C::KL, KU = C::KU, NB = BC::NB;
    constexpr int IB = BC::IB, H = BC::H, IBO = BC::IBO;
    constexpr int ROWB = IB * 16, ROWBO = IBO * 16;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t crank = cluster_ctarank();

    double* table = reinterpret_cast<double*>(smem_raw);
    double* scratch = reinterpret_cast<double*>(smem_raw + BC::TBL);
    double* xchg = scratch + W * kScratchPerWarp;  // 2 parities x XN doubles
    uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(xchg) + C::XCHG);
    unsigned char* after = reinterpret_cast<unsigned char*>(bars + 4);
    const uint32_t pad = (1024u - (smem_u32(after) & 1023u)) & 1023u;
    unsigned char* buf0 = after + pad;
    unsigned char* buf1 = buf0 + BC::BUF;
    const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
    const uint32_t cbar = smem_u32(&bars[2]);
    volatile int* cflag = reinterpret_cast<volatile int*>(&bars[3]);
    uint32_t cphase = 0;

    if (threadIdx.x < 2) mbar_init(smem_u32(&bars[threadIdx.x]), W);
    if (threadIdx.x == 2) mbar_init(cbar, C::C);
    mbar_init_fence();
    // Every CTA of the cluster has started and initialised its mbarriers
    // before any CTA arrives on a peer's (the one hardware cluster barrier,
    // which every CTA reaches).
    cluster_sync();
    bool alive = cl_prologue<C>(op, table, scratch, xchg, crank, cbar, cphase, cflag);
    __syncthreads();
    if (!alive && threadIdx.x == 0) atomicOr(&g_stream_status, kStatusWaitTimeout | kStatusClusterBarrier);

    GroupCtx g;
    g.lane = lane;
    g.wg = warp;
    g.W = W;
    g.nthr = T;
    g.bar_id = 1;
    g.seq = 0;
    g.scratch = scratch;

    const int t = threadIdx.x;
    const int64_t s_glob = (int64_t)crank * C::S + (int64_t)t * R;
    const double2* tb = reinterpret_cast<const double2*>(table) + t;
    auto coef = [&](int p, int u) -> double2 { return tb[(p * U + u) * BC::TP]; };
    double Af = 1.0, Ab = 1.0;
    if constexpr (BC::FWD) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const double2 c = coef(BC::P_NL, u);
            Af = (u == 0) ? c.x : c.x * Af;
            Af = c.y * Af;
        }
    }
    if constexpr (BC::BWD) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const double2 c = coef(BC::P_NH, u);
            Ab = c.x * Ab;
            Ab = c.y * Ab;
        }
    }
    const int sw_me = swz_row<BC::SWB>(t), sw_prev = swz_row<BC::SWB>(t - 1), sw_next = swz_row<BC::SWB>(t + 1);
    const int sw_lastc = swz_row<BC::SWB>(T - 1), sw_firstc = swz_row<BC::SWB>(0);
    const int swo_me = swz_row<BC::SWBO>(t);
    auto unit_off = [&](int u, int c, int sw) -> uint32_t {
        return (uint32_t)((H > 1 ? (u / IB) * T : 0) + c) * ROWB + (((u % IB) ^ sw) << 4);
    };

    const bool win_partial = io.iz0 > 0 || io.iz1 < io.M;
    const int64_t nsys = io.nsys;
    const int64_t step = num_clusters_x();
    int64_t sys = cluster_id_x();
    const int chunk0 = (int)crank * T;  // this CTA's first chunk

    auto issue_load = [&](unsigned char* b, uint32_t bar, int64_t y) {
        mbar_arrive_expect_tx(bar, (uint32_t)(H * 32 * ROWB));
#pragma unroll
        for (int h = 0; h < H; ++h)
            tma_load_3d(smem_u32(b + (size_t)(h * T + 32 * warp) * ROWB), &tm_in, h * IB * 2, chunk0 + 32 * warp, (int)y,
                        bar);
    };
    auto issue_store = [&](unsigned char* b, int64_t y) {
#pragma unroll
        for (int h = 0; h < BC::HO; ++h)
            tma_store_3d(&tm_out, h * IBO * 2, chunk0 + 32 * warp, (int)y,
                         smem_u32(b + (size_t)(h * T + 32 * warp) * ROWBO));
        bulk_commit();
    };

    if (!alive) sys = nsys;
    if (sys < nsys && lane == 0) issue_load(buf0, bar0, sys);
    // A failed TMA wait (bits 0) stops every CTA at the same point, and the
    // final barrier still runs; a cluster barrier that ran out (alive = false)
    // skips it, since a peer that never arrived will not arrive there either.
    auto stop = [&](unsigned bits) {
        if (t == 0) atomicOr(&g_stream_status, kStatusWaitTimeout | bits);
        if (bits) alive = false;
    };
    // Waits for the TMA load of the k-th system of this cluster and publishes
    // the outcome for the peers.  It is published before a cluster barrier --
    // the first one for k = 0, otherwise the last one of system k-1 -- after
    // which the system's rows are readable by every CTA and all CTAs read the
    // same outcomes.
    auto wait_publish = [&](int k) {
        bool ok = mbar_wait_bounded((k & 1) ? bar1 : bar0, (uint32_t)((k >> 1) & 1));
        ok = group_and(g.bar_id, g.nthr, ok);
        if (t == 0) xchg[(k & 1) * C::XN + C::XOK] = ok ? 1.0 : 0.0;
    };
    if (sys < nsys) {
        wait_publish(0);
        if (!cl_barrier<C::C>(cbar, cphase, cflag, T)) {
            stop(kStatusClusterBarrier << 1);
            sys = nsys;
        }
    }
    for (int k = 0; sys < nsys; ++k, sys += step) {
        unsigned char* cur = (k & 1) ? buf1 : buf0;
        unsigned char* nxt = (k & 1) ? buf0 : buf1;
        double* xc = xchg + (k & 1) * C::XN;
        const bool more = sys + step < nsys;
        {
            bool a = true;
            for (uint32_t r = 0; r < C::C; ++r) a = a && ld_cluster_f64(mapa_rank(smem_u32(xc + C::XOK), r)) != 0.0;
            if (!a) {
                stop(0);
                break;
            }
        }

        double be[R + KL + KU];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const double2 v = *reinterpret_cast<const double2*>(cur + unit_off(u, t, sw_me));
            be[KL + 2 * u] = v.x;
            be[KL + 2 * u + 1] = v.y;
        }
        if constexpr (KL > 0) {
            double2 pv = make_double2(0.0, 0.0);
            if (t > 0) {
                pv = *reinterpret_cast<const double2*>(cur + unit_off(U - 1, t - 1, sw_prev));
            } else if (crank > 0) {
                pv = ld_cluster_v2(mapa_rank(smem_u32(cur + unit_off(U - 1, T - 1, sw_lastc)), crank - 1));
            }
            be[KL - 1] = pv.y;
            if constexpr (KL > 1) be[0] = pv.x;
        }
        if constexpr (KU > 0) {
            double2 nv = make_double2(0.0, 0.0);
            if (t < T - 1) {
                nv = *reinterpret_cast<const double2*>(cur + unit_off(0, t + 1, sw_next));
            } else if (crank + 1 < (uint32_t)C::C) {
                nv = ld_cluster_v2(mapa_rank(smem_u32(cur + unit_off(0, 0, sw_firstc)), crank + 1));
            }
            be[KL + R] = nv.x;
            if constexpr (KU > 1) be[KL + R + 1] = nv.y;
        }
        if (win_partial) {
#pragma unroll
            for (int i = 0; i < R + KL + KU; ++i) {
                const int64_t row = s_glob - KL + i;
                if (row < io.iz0 || row >= io.iz1) be[i] = 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            double2 wc[NB];
#pragma unroll
            for (int q = 0; q < NB; ++q) wc[q] = coef(q, u);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int j = 2 * u + e;
                double acc = (e ? wc[0].y : wc[0].x) * be[j];
#pragma unroll
                for (int q = 1; q < NB; ++q) acc = __fma_rn(e ? wc[q].y : wc[q].x, be[j + q], acc);
                be[j] = acc;
            }
        }
        double (&x)[R + KL + KU] = be;
        if (more && lane == 0) {
            bulk_wait_read_all();
            issue_load(nxt, (k & 1) ? bar0 : bar1, sys + step);
        }

        if constexpr (BC::FWD) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const double2 c = coef(BC::P_NL, u);
                if (u > 0) x[2 * u] = __fma_rn(c.x, x[2 * u - 1], x[2 * u]);
                x[2 * u + 1] = __fma_rn(c.y, x[2 * u], x[2 * u + 1]);
            }
            double Ain, Bin, At, Bt;
            group_affine_scan_map<true>(g, Af, x[R - 1], Ain, Bin, At, Bt);
            if (t == T - 1) {
                xc[C::XF] = At;
                xc[C::XF + 1] = Bt;
            }
            if (!BC::BWD && more) wait_publish(k + 1);
            if (!cl_barrier<C::C>(cbar, cphase, cflag, T)) {
                stop(kStatusClusterBarrier << 2);
                break;
            }
            double X = 0.0;  // value entering this CTA's slice
            for (uint32_t r = 0; r < crank; ++r) {
                const uint32_t ra = mapa_rank(smem_u32(xc + C::XF), r);
                X = __fma_rn(ld_cluster_f64(ra), X, ld_cluster_f64(ra + 8));
            }
            const double pin = __fma_rn(Ain, X, Bin);
            double p = 1.0;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const double2 c = coef(BC::P_NL, u);
                p = c.x * p;
                x[2 * u] = __fma_rn(p, pin, x[2 * u]);
                p = c.y * p;
                x[2 * u + 1] = __fma_rn(p, pin, x[2 * u + 1]);
            }
        }
        if constexpr (BC::BWD) {
#pragma unroll
            for (int u = U - 1; u >= 0; --u) {
                const double2 c = coef(BC::P_NH, u);
                if (u < U - 1) x[2 * u + 1] = __fma_rn(c.y, x[2 * u + 2], x[2 * u + 1]);
                x[2 * u] = __fma_rn(c.x, x[2 * u + 1], x[2 * u]);
            }
            double Ain, Bin, At, Bt;
            group_affine_scan_map<false>(g, Ab, x[0], Ain, Bin, At, Bt);
            if (t == 0) {
                xc[C::XB] = At;
                xc[C::XB + 1] = Bt;
            }
            if (more) wait_publish(k + 1);
            if (!cl_barrier<C::C>(cbar, cphase, cflag, T)) {
                stop(kStatusClusterBarrier << 3);
                break;
            }
            double X = 0.0;  // value entering this CTA's slice from above
            for (uint32_t r = C::C - 1; r > crank; --r) {
                const uint32_t ra = mapa_rank(smem_u32(xc + C::XB), r);
                X = __fma_rn(ld_cluster_f64(ra), X, ld_cluster_f64(ra + 8));
            }
            const double q = __fma_rn(Ain, X, Bin);
            double p = 1.0;
#pragma unroll
            for (int u = U - 1; u >= 0; --u) {
                const double2 c = coef(BC::P_NH, u);
                p = c.y * p;
                x[2 * u + 1] = __fma_rn(p, q, x[2 * u + 1]);
                p = c.x * p;
                x[2 * u] = __fma_rn(p, q, x[2 * u]);
            }
        }
        if (C::SV != SV_NONE && s_glob == 0) x[0] = op.scaleC * x[0];
        // In place: the neighbour CTAs read this slice's halo rows before the
        // scans' cluster barriers; without a solve, wait for them here.
        if constexpr (C::SV == SV_NONE) {
            if (more) wait_publish(k + 1);
            if (!cl_barrier<C::C>(cbar, cphase, cflag, T)) {
                stop(kStatusClusterBarrier << 4);
                break;
            }
        }
        __syncwarp();
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int h = u / IBO, uu = u % IBO;
            *reinterpret_cast<double2*>(cur + (size_t)(h * T + t) * ROWBO + ((uu ^ swo_me) << 4)) =
                make_double2(x[2 * u], x[2 * u + 1]);
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) issue_store(cur, sys);
    }
    if (lane == 0) bulk_wait_all();
    // No CTA leaves while a peer may still read its shared memory.
    if (alive && !cl_barrier<C::C>(cbar, cphase, cflag, T)) stop(kStatusClusterBarrier << 5);
}

}  // namespace pfb
