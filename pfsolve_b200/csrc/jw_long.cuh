// jw_long.cuh -- the JW step for long systems (N > 4096) in two passes, with
// no waiting between CTAs.
//
// Same operator as the streaming and cluster kernels (x = M^{-1} V b,
// x[0] *= scaleC; real FP64 systems; PfSolve_shaderGen_JonesWorlandMV,
// pfSolve_CodeGen/pfSolve_KernelsLevel2/pfSolve_JonesWorland.h:38-408).  The
// reference splits such systems over several launches that keep a reduced
// system in a temporary buffer (multi-upload,
// pfSolve_AppManagement/pfSolve_InitializeApp.h:1540-1583); so does this
// kernel, with the reduction written as affine maps:
//
//  * A system is cut into NS slices of S = 32*W*R rows.  In the solve passes a
//    CTA takes an even share of the (slice, system) items in slice-major
//    order -- one slice or a few, whose coefficient tables it loads into
//    shared memory in turn -- and G groups of W warps each stream a different
//    system's slice through the table (TMA boxes, as in the streaming kernel).
//  * Within a slice the solve is the group kernel's: per-thread chunk
//    recurrences and affine scans across the group.  The value entering the
//    slice from below (forward) or above (backward) is the only coupling.
//  * Two table passes, one CTA per slice, build every slice's coefficient
//    table once per launch: the first (PASS = 3, tridiagonal solves only)
//    writes the Moebius product of each slice's pivot recurrence, the second
//    (PASS = 0) composes those of the slices below it -- the pivot entering
//    the slice -- builds the table and writes it, with the slice's constants
//    (below), to global memory; the two solve passes copy their slice's
//    table from there.
//  * Pass 1 (PASS = 1) needs, per (system, slice), only the slice's offsets
//    with both carries zero: the forward offset Bf (the value leaving the
//    slice) and the backward offset Bb0.  Both are linear in the matvec result
//    g of the slice's rows -- Bf = sum alpha_k g_k, Bb0 = sum beta_k g_k with
//    alpha_k the product of the forward solve band over rows k+1.., gamma_i
//    that of the backward band over rows ..i-1 and beta_k = gamma_k +
//    nl_{k+1} beta_{k+1} -- so pass 1 is the matvec and two reductions, with
//    alpha and beta formed once per launch by the table pass.  It writes them
//    and the slice's matvec halo input rows (so pass 2 never reads rows a neighbour slice may already have
//    overwritten in place).  The slice constants of the table pass: the
//    forward and backward multipliers Af, Ab, and Psi, the backward offset for
//    a unit forward carry and zero input (the backward offset is affine in the
//    forward carry: Bb = Bb0 + X Psi).
//  * Between the passes a small kernel (one thread per system) composes the
//    forward carries X_c = Af_{c-1} X_{c-1} + Bf_{c-1} from slice 0 and the
//    backward ones from the top slice, Y_c = Ab_{c+1} Y_{c+1} + Bb0_{c+1} +
//    X_{c+1} Psi_{c+1}, into the records.
//  * Pass 2 solves its slice again with those carries and writes the result.
//  Input is read twice and written once; the four launches are ordered on
//  the stream, so no CTA ever waits for another.
//  * The single-pass form (PASS = 4, the default) reads the input once: after
//    the two table passes, one cooperative launch (every CTA resident) solves
//    each slice with zero carries, publishes the slice's offsets (Bf, Bb0)
//    with a release flag, waits for the other slices of the same system
//    (acquire loads of their flags, bounded), composes the carries entering
//    its slice from the published offsets and the slice constants, and adds
//    their responses: x = x0 + X psi + Y G, with psi (a unit forward carry,
//    zero input) and G (a unit backward carry) per row, built once per CTA.
//    All slices of a system are handled by the same group index of the CTAs
//    of one column (CTA b: slice b % NS, column b / NS), which take the
//    systems in the same order, so every wait is on groups that are resident
//    and about to publish.  A slice reads its matvec halo rows from global
//    memory before publishing, and no slice of a system stores before all of
//    them have published: in place is safe.
//  * Completion waits are bounded: a wait that runs out records
//    kStatusWaitTimeout and the group stops.
#pragma once
#include "jw_cluster.cuh"

namespace pfb {

template <int R_, int W_, int G_, int KL_, int KU_, int SV_>
struct LgCfg {
    using B = StCfg<R_, W_, KL_, KU_, SV_, LAY_REAL, LAY_REAL, false, PREC_F64, 0, 0>;  // slice layout and table planes
    static constexpr int R = R_, W = W_, G = G_, T = 32 * W_, S = T * R_, NT = T * G_;
    static constexpr int KL = KL_, KU = KU_, SV = SV_;
};

// Per (system, slice) record, in doubles: forward offset and backward offset
// (pass 1), halo rows below (KL <= 2) and above (KU <= 2) (pass 1), and the
// carries entering the slice from below and from above (the carry kernel).
// Stored slice-major, field k of system y in slice c at (c * kLgRed + k) *
// nsys + y, so that the carry kernel's threads (one per system) read
// consecutive addresses.
constexpr int kLgRed = 8;
constexpr int kLgRedBf = 0, kLgRedBb = 1, kLgRedLo = 2, kLgRedHi = 4, kLgRedX = 6, kLgRedY = 7;
// Per slice constants: Af, Ab, Psi, then the Moebius product of the slice's
// rows (tridiagonal pivots; 4 doubles at kLgConstMob).
constexpr int kLgConst = 8;
constexpr int kLgConstMob = 4;
// Slices per system the single-pass form composes (two rounds of a warp).
constexpr int kLgMaxSlices = 64;
// Cross-CTA waits of the single-pass form give up after this many cycles
// (about 0.5 s at the B200's clock).
constexpr long long kLgWaitCycles = 1000000000LL;

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Staging buffers per group: two (a system in flight ahead of the one being
// solved), three in the single pass (its phase B trails phase A by a system).
template <int PASS>
struct LgBufs {
    static constexpr int v = PASS == 4 ? 3 : 2;
};

// Shared memory: table | scratch | 8 doubles | slice constants (Af, Ab, Psi
// of up to kLgMaxSlices slices, 4 doubles each) | mbarriers | (align 1024) |
// buffers | per row of the slice, 16 bytes: the PASS 1 weights (alpha, beta),
// or in the single pass the carry responses (psi, G) | in the solve passes,
// two slots of R doubles per group for a last partial chunk.
template <class C, int NBUF = 2>
__host__ __device__ constexpr size_t lg_smem_bytes()
{
    return C::B::TBL + (size_t)C::G * C::W * kScratchPerWarp * sizeof(double) + 8 * sizeof(double) +
           (size_t)kLgMaxSlices * 4 * sizeof(double) + (size_t)C::G * NBUF * sizeof(uint64_t) + 1024 +
           (size_t)C::G * NBUF * C::B::BUF + (size_t)C::S * 16 +
           (NBUF == 2 ? (size_t)C::G * 2 * C::R * sizeof(double) : 0);  // the solve passes' tail slots
}

// ---- Coefficient table of slice c (rows c*S + [0, S)), built by all threads
// of the CTA; the pivots entering the slice come from the Moebius products
// of the slices below it (cst, written by the PASS = 3 launch).  With
// AGG_ONLY the CTA instead writes its own slice's product there.
template <class C, bool AGG_ONLY = false>
__device__ void lg_prologue(const JwOperator& op, double* table, double* scratch, double* q4, int c,
                            double* __restrict__ cst)
{
    using BC = typename C::B;
    constexpr int R = C::R, U = BC::U, NB = BC::NB, S = C::S;
    const int64_t M = op.M;
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int64_t s0 = (int64_t)c * S;  // first row of the slice
    GroupCtx g;
    g.lane = tid & 31;
    g.wg = tid >> 5;
    g.W = nthr >> 5;
    g.nthr = nthr;
    g.bar_id = 1;
    g.seq = 0;
    g.scratch = scratch;
    auto mstep = [&](int64_t i, double& a, double& b, double& cc, double& d) {
        double ac = 0.0;
        if (i >= 1 && i < M) ac = band(op, op.off_sl, i) * band(op, op.off_su, i - 1);
        const double na = a - ac * cc, nb = b - ac * d;
        cc = a;
        d = b;
        a = na;
        b = nb;
        renorm2x2(a, b, cc, d);
    };
    double dprev = 1.0;
    const int Rp = (S + nthr - 1) / nthr;
    const int64_t s = s0 + (int64_t)tid * Rp;
    if constexpr (C::SV == SV_TRI) {
        // this thread's rows of the slice, then the product of the slice's
        // preceding chunks
        double a = 1, b = 0, cc = 0, d = 1;
        for (int j = 0; j < Rp; ++j) {
            const int64_t i = s + j;
            if (i < s0 + S) mstep(i, a, b, cc, d);
        }
        const double pa = a, pb = b, pc = cc, pd = d;
        group_matrix_scan(g, a, b, cc, d);
        if constexpr (AGG_ONLY) {
            // the slice's product = last thread's own * its preceding
            if (tid == nthr - 1) {
                double na = pa * a + pb * cc, nb = pa * b + pb * d, nc = pc * a + pd * cc, nd = pc * b + pd * d;
                renorm2x2(na, nb, nc, nd);
                double* o = cst + c * kLgConst + kLgConstMob;
                o[0] = na;
                o[1] = nb;
                o[2] = nc;
                o[3] = nd;
            }
            return;
        }
        // Q = product of the slices below: agg[c-1] * ... * agg[0], the
        // products loaded in blocks of 8 ahead of their chain
        double qa = 1, qb = 0, qc = 0, qd = 1;
        for (int r0 = 0; r0 < c; r0 += 8) {
            double4 m[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const double* o = cst + (r0 + q) * kLgConst + kLgConstMob;
                m[q] = (r0 + q < c) ? make_double4(o[0], o[1], o[2], o[3]) : make_double4(1.0, 0.0, 0.0, 1.0);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                if (r0 + q >= c) break;
                double na = m[q].x * qa + m[q].y * qc, nb = m[q].x * qb + m[q].y * qd, nc = m[q].z * qa + m[q].w * qc,
                       nd = m[q].z * qb + m[q].w * qd;
                renorm2x2(na, nb, nc, nd);
                qa = na;
                qb = nb;
                qc = nc;
                qd = nd;
            }
        }
        (void)q4;
        // full prefix = (slice prefix) * Q; incoming vector = prefix * (1, 0)^T
        const double fa = a * qa + b * qc, fc = cc * qa + d * qc;
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
}

// One slice solve of a group: x holds the matvec result on entry and the
// slice's solution on exit.  Carries: fwd_carry(Atot, Btot) returns the value
// entering the slice from below given the slice's forward total map;
// bwd_carry likewise from above.  Both are called by every thread of the group.
template <class C, class TB, class FC, class BCR>
__device__ __forceinline__ void lg_solve(GroupCtx& g, const TB& coef, double Af, double Ab, double (&x)[C::R + C::KL + C::KU],
                                         FC fwd_carry, BCR bwd_carry)
{
    using BC = typename C::B;
    constexpr int R = C::R, U = BC::U;
    (void)R;
    if constexpr (BC::FWD) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const double2 c = coef(BC::P_NL, u);
            if (u > 0) x[2 * u] = __fma_rn(c.x, x[2 * u - 1], x[2 * u]);
            x[2 * u + 1] = __fma_rn(c.y, x[2 * u], x[2 * u + 1]);
        }
        double Ain, Bin, At, Bt;
        group_affine_scan_map<true>(g, Af, x[C::R - 1], Ain, Bin, At, Bt);
        const double X = fwd_carry(At, Bt);
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
        const double Y = bwd_carry(At, Bt);
        const double q = __fma_rn(Ain, Y, Bin);
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
}

// Carries of every slice of system blockIdx.x * blockDim.x + threadIdx.x.
template <bool FWD, bool BWD>
__global__ void __launch_bounds__(128) jw_long_carry_kernel(double* __restrict__ red, const double* __restrict__ cst,
                                                            const int NS, const int64_t nsys)
{
    const int64_t y = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= nsys) return;
    auto rs = [&](int c, int k) -> double& { return red[((size_t)c * kLgRed + k) * nsys + y]; };
    // slices in blocks of B, each block's loads issued together ahead of its
    // dependent chain of FMAs
    constexpr int B = 8;
    double X = 0.0;
    for (int c0 = 0; c0 < NS; c0 += B) {
        double bf[B], af[B];
#pragma unroll
        for (int q = 0; q < B; ++q) {
            const bool v = FWD && c0 + q < NS;
            bf[q] = v ? rs(c0 + q, kLgRedBf) : 0.0;
            af[q] = v ? cst[(c0 + q) * kLgConst] : 1.0;
        }
#pragma unroll
        for (int q = 0; q < B; ++q) {
            if (c0 + q >= NS) break;
            rs(c0 + q, kLgRedX) = X;
            if (FWD) X = __fma_rn(af[q], X, bf[q]);
        }
    }
    if (BWD) {
        double Y = 0.0;
        for (int c0 = ((NS - 1) / B) * B; c0 >= 0; c0 -= B) {
            double bb[B], ab[B];
#pragma unroll
            for (int q = 0; q < B; ++q) {
                const int c = c0 + q;
                bb[q] = 0.0;
                ab[q] = 1.0;
                if (c < NS) {
                    bb[q] = FWD ? __fma_rn(rs(c, kLgRedX), cst[c * kLgConst + 2], rs(c, kLgRedBb)) : rs(c, kLgRedBb);
                    ab[q] = cst[c * kLgConst + 1];
                }
            }
#pragma unroll
            for (int q = B - 1; q >= 0; --q) {
                if (c0 + q >= NS) continue;
                rs(c0 + q, kLgRedY) = Y;
                Y = __fma_rn(ab[q], Y, bb[q]);
            }
        }
    }
}


// Carries entering slice c of system y in the single pass (called by the 32
// lanes of one warp once every slice of y has published): X from below, the
// maps (Af, Bf) of the slices composed upwards; Y from above, the maps
// (Ab, Bb0 + X Psi) composed downwards.  Lanes hold slices, in rounds of 32.
// Returns the carries on every lane.
template <bool FWD, bool BWD>
__device__ __forceinline__ void lg_compose(int lane, int c, int NS, int64_t nsys, int64_t y,
                                           const double* __restrict__ red, const double* cst_s, double& Xin,
                                           double& Yin)
{
    double Xr[kLgMaxSlices / 32];
    double carry = 0.0;
    Xin = 0.0;
    Yin = 0.0;
#pragma unroll
    for (int r = 0; r < kLgMaxSlices / 32; ++r) {
        Xr[r] = 0.0;
        if (32 * r >= NS) break;  // no slices left (NS is uniform)
        const int cc = 32 * r + lane;
        const bool v = cc < NS && FWD;
        double A = v ? cst_s[4 * cc] : 1.0;
        double B = v ? __ldcg(&red[((size_t)cc * kLgRed + kLgRedBf) * nsys + y]) : 0.0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {  // inclusive scan of the maps
            const double Ap = __shfl_up_sync(FULL, A, d), Bp = __shfl_up_sync(FULL, B, d);
            if (lane >= d) {
                B = __fma_rn(A, Bp, B);
                A = A * Ap;
            }
        }
        const double incl = __fma_rn(A, carry, B);  // value leaving slice cc
        double ex = __shfl_up_sync(FULL, incl, 1);
        if (lane == 0) ex = carry;
        Xr[r] = ex;  // value entering slice cc
        if (cc == c) Xin = ex;
        carry = __shfl_sync(FULL, incl, 31);
    }
    if constexpr (BWD) {
        carry = 0.0;
#pragma unroll
        for (int r = kLgMaxSlices / 32 - 1; r >= 0; --r) {
            if (32 * r >= NS) continue;  // identity maps above the top slice
            const int cc = 32 * r + lane;
            const bool v = cc < NS;
            double A = v ? cst_s[4 * cc + 1] : 1.0;
            double B = v ? __fma_rn(Xr[r], cst_s[4 * cc + 2], __ldcg(&red[((size_t)cc * kLgRed + kLgRedBb) * nsys + y]))
                         : 0.0;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {  // inclusive scan from the top
                const double Ap = __shfl_down_sync(FULL, A, d), Bp = __shfl_down_sync(FULL, B, d);
                if (lane + d < 32) {
                    B = __fma_rn(A, Bp, B);
                    A = A * Ap;
                }
            }
            const double incl = __fma_rn(A, carry, B);  // value leaving slice cc downwards
            double ex = __shfl_down_sync(FULL, incl, 1);
            if (lane == 31) ex = carry;
            if (cc == c) Yin = ex;
            carry = __shfl_sync(FULL, incl, 0);
        }
    }
    const int owner = c & 31;  // the lane of slice c holds its carries
    Xin = __shfl_sync(FULL, Xin, owner);
    Yin = __shfl_sync(FULL, Yin, owner);
}

// PASS 3: grid NS (CTA c writes slice c's pivot product into cst, tridiagonal
// only); PASS 0: grid NS (CTA c builds slice c's table into tab + c * TBL / 8
// and its constants into cst); PASS 1, 2 and 4 (the single pass, a
// cooperative launch): CTAs in multiples of NS (CTA b owns slice b % NS).
// red: io.nsys * NS records of kLgRed doubles; cst: NS records of kLgConst
// doubles; flags (single pass): io.nsys * NS words, slice-major, set to
// `epoch` when a (system, slice) record is published.
template <class C, int PASS>
__global__ void __launch_bounds__(C::NT) jw_long_kernel(const __grid_constant__ CUtensorMap tm_in,
                                                       const __grid_constant__ CUtensorMap tm_out,
                                                       const JwOperator op, const JwIO io, double* __restrict__ red,
                                                       double* __restrict__ cst, double* __restrict__ tab,
                                                       const int NS, unsigned* __restrict__ flags,
                                                       const unsigned epoch)
{
    using BC = typename C::B;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int R = C::R, W = C::W, T = C::T, U = BC::U, KL = C::KL, KU = C::KU, NB = BC::NB;
    constexpr int IB = BC::IB, H = BC::H, IBO = BC::IBO;
    constexpr int ROWB = IB * 16, ROWBO = IBO * 16;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = warp / W, wg = warp - grp * W;
    const int t = threadIdx.x - grp * T;  // thread within the group
    // Passes 1 and 2 take a range of the slice-major list of (slice, system)
    // items -- CTA b: [b L, (b+1) L), L = ceil(NS nsys / grid) -- so that every
    // CTA of the grid has work whatever NS; a range spans one slice or a few,
    // and the CTA loads each one's table in turn.  The other passes: CTA b
    // owns slice b % NS.
    int64_t it_beg = 0, it_end = 0;
    int c = (int)(blockIdx.x % (unsigned)NS);
    if constexpr (PASS == 1 || PASS == 2) {
        const int64_t total = (int64_t)NS * io.nsys;
        const int64_t L = (total + gridDim.x - 1) / gridDim.x;
        it_beg = (int64_t)blockIdx.x * L < total ? (int64_t)blockIdx.x * L : total;
        it_end = it_beg + L < total ? it_beg + L : total;
        c = it_beg < it_end ? (int)(it_beg / io.nsys) : 0;
    }

    double* table = reinterpret_cast<double*>(smem_raw);
    double* scratch = reinterpret_cast<double*>(smem_raw + BC::TBL);
    double* q4 = scratch + C::G * W * kScratchPerWarp;  // 8 doubles
    double* cst_s = q4 + 8;                              // slice constants (single pass)
    uint64_t* bars_all = reinterpret_cast<uint64_t*>(cst_s + kLgMaxSlices * 4);
    uint64_t* bars = bars_all + LgBufs<PASS>::v * grp;
    constexpr int NBUF = LgBufs<PASS>::v;
    unsigned char* after = reinterpret_cast<unsigned char*>(bars_all + NBUF * C::G);
    const uint32_t pad = (1024u - (smem_u32(after) & 1023u)) & 1023u;
    unsigned char* buf0 = after + pad + (size_t)grp * NBUF * BC::BUF;
    unsigned char* buf1 = buf0 + BC::BUF;
    // PASS 1 weights: row tt * R + jj at [jj * T + tt] (consecutive threads,
    // consecutive entries)
    double2* ab_s = reinterpret_cast<double2*>(after + pad + (size_t)C::G * NBUF * BC::BUF);
    // solve passes: this group's two slots for a last partial chunk of R rows
    double* tail_s = reinterpret_cast<double*>(ab_s + C::S) + (size_t)grp * 2 * R;
    auto ab_g_of = [&](int cc) -> double2* {
        return reinterpret_cast<double2*>(tab + (size_t)NS * (BC::TBL / sizeof(double))) + (size_t)cc * C::S;
    };
    double2* ab_g = ab_g_of(c);
    const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);

    if (threadIdx.x < NBUF * C::G) mbar_init(smem_u32(bars_all + threadIdx.x), W);
    mbar_init_fence();
    double* gtab = tab + (size_t)c * (BC::TBL / sizeof(double));
    // the solve passes' copy of slice c's table (and pass 1's weights)
    auto load_slice = [&]() {
        const double2* src = reinterpret_cast<const double2*>(tab + (size_t)c * (BC::TBL / sizeof(double)));
        double2* dst = reinterpret_cast<double2*>(table);
        for (int i = threadIdx.x; i < (int)(BC::TBL / 16); i += blockDim.x) dst[i] = src[i];
        if constexpr (PASS == 1) {
            const double2* w = ab_g_of(c);
            for (int i = threadIdx.x; i < C::S; i += blockDim.x) ab_s[i] = w[i];
        }
    };
    if constexpr (PASS == 3) {
        lg_prologue<C, true>(op, table, scratch, q4, c, cst);
        return;
    } else if constexpr (PASS == 0) {
        lg_prologue<C>(op, table, scratch, q4, c, cst);
    } else {
        load_slice();
        if constexpr (PASS == 4)
            for (int i = threadIdx.x; i < NS; i += blockDim.x) {
                cst_s[4 * i] = cst[i * kLgConst];          // Af
                cst_s[4 * i + 1] = cst[i * kLgConst + 1];  // Ab
                cst_s[4 * i + 2] = cst[i * kLgConst + 2];  // Psi
            }
    }
    __syncthreads();

    GroupCtx g;
    g.lane = lane;
    g.wg = wg;
    g.W = W;
    g.nthr = T;
    g.bar_id = 1 + grp;
    g.seq = 0;
    g.scratch = scratch + (size_t)grp * W * kScratchPerWarp;

    int64_t s0 = (int64_t)c * C::S;
    int64_t s_glob = s0 + (int64_t)t * R;
    const double2* tb = reinterpret_cast<const double2*>(table) + t;
    auto coef = [&](int p, int u) -> double2 { return tb[(p * U + u) * BC::TP]; };
    double Af = 1.0, Ab = 1.0;  // this thread's chunk multipliers
    auto chunk_mults = [&]() {
        Af = 1.0;
        Ab = 1.0;
        if constexpr (BC::FWD) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const double2 cc = coef(BC::P_NL, u);
                Af = (u == 0) ? cc.x : cc.x * Af;
                Af = cc.y * Af;
            }
        }
        if constexpr (BC::BWD) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const double2 cc = coef(BC::P_NH, u);
                Ab = cc.x * Ab;
                Ab = cc.y * Ab;
            }
        }
    };
    chunk_mults();

    // Single pass: the responses of the slice's rows to a unit forward carry
    // (psi) and to a unit backward carry (G), by group 0: zero-input solves.
    if constexpr (PASS == 4) {
        if (grp == 0) {
            double xp[R + KL + KU], xg[R + KL + KU];
#pragma unroll
            for (int i = 0; i < R + KL + KU; ++i) {
                xp[i] = 0.0;
                xg[i] = 0.0;
            }
            lg_solve<C>(g, coef, Af, Ab, xp, [&](double, double) { return 1.0; }, [&](double, double) { return 0.0; });
            lg_solve<C>(g, coef, Af, Ab, xg, [&](double, double) { return 0.0; }, [&](double, double) { return 1.0; });
#pragma unroll
            for (int j = 0; j < R; ++j) ab_s[j * T + t] = make_double2(xp[j], xg[j]);
        }
        __syncthreads();
    }
    // Slice constants (Af, Ab, Psi): a solve of zero input with a unit
    // forward carry, by group 0, and the table itself to global memory.
    if constexpr (PASS == 0) {
        double2* dst = reinterpret_cast<double2*>(gtab);
        const double2* src = reinterpret_cast<const double2*>(table);
        for (int i = threadIdx.x; i < (int)(BC::TBL / 16); i += blockDim.x) dst[i] = src[i];
    }
    if (PASS == 0 && grp == 0) {
        double x[R + KL + KU];
#pragma unroll
        for (int i = 0; i < R + KL + KU; ++i) x[i] = 0.0;
        double afs = 1.0, abs_ = 1.0, psi = 0.0;
        lg_solve<C>(g, coef, Af, Ab, x,
                    [&](double At, double) {
                        afs = At;
                        return 1.0;
                    },
                    [&](double At, double Bt) {
                        abs_ = At;
                        psi = Bt;
                        return 0.0;
                    });
        if (t == 0) {
            cst[c * kLgConst + 0] = afs;
            cst[c * kLgConst + 1] = abs_;
            cst[c * kLgConst + 2] = psi;
        }
    }
    if constexpr (PASS == 0) {
        // PASS 1 weights of the slice, by group 0 (thread t: rows tR .. tR+R-1):
        // gamma by a forward product scan, alpha by a backward product scan,
        // beta by a backward affine scan of beta_k = gamma_k + nl_{k+1} beta_{k+1}
        if (grp == 0) {
            double nlv[R], nhv[R];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const double2 l2 = BC::FWD ? coef(BC::P_NL, u) : make_double2(0.0, 0.0);
                const double2 h2 = BC::BWD ? coef(BC::P_NH, u) : make_double2(1.0, 1.0);
                nlv[2 * u] = l2.x;
                nlv[2 * u + 1] = l2.y;
                nhv[2 * u] = h2.x;
                nhv[2 * u + 1] = h2.y;
            }
            double Ain, Bin, At, Bt;
            double P = 1.0;
#pragma unroll
            for (int j = 0; j < R; ++j) P *= nhv[j];
            group_affine_scan_map<true>(g, P, 0.0, Ain, Bin, At, Bt);
            double gam[R];
            double cur = Ain;  // product of the preceding chunks' bands
#pragma unroll
            for (int j = 0; j < R; ++j) {
                gam[j] = cur;
                cur *= nhv[j];
            }
            P = 1.0;
#pragma unroll
            for (int j = 0; j < R; ++j) P *= nlv[j];
            double Aa, Ba, At2, Bt2;
            group_affine_scan_map<false>(g, P, 0.0, Aa, Ba, At2, Bt2);  // Aa: product of the later chunks' bands
            // nl of the next chunk's first row (0 past the slice)
            const double nl_after = (BC::FWD && t + 1 < T) ? tb[(BC::P_NL * U) * BC::TP + 1].x : 0.0;
            double A = 1.0, Bl = 0.0;  // this chunk's beta map, entering value = beta of row (t+1)R
#pragma unroll
            for (int k = R - 1; k >= 0; --k) {
                const double nn = (k == R - 1) ? nl_after : nlv[k + 1];
                Bl = __fma_rn(nn, Bl, gam[k]);
                A *= nn;
            }
            double Ab2, Bb2, At3, Bt3;
            group_affine_scan_map<false>(g, A, Bl, Ab2, Bb2, At3, Bt3);
            double beta = Bb2, alpha = Aa;  // entering this chunk from above (slice input 0)
#pragma unroll
            for (int k = R - 1; k >= 0; --k) {
                const double nn = (k == R - 1) ? nl_after : nlv[k + 1];
                beta = __fma_rn(nn, beta, gam[k]);
                if (k < R - 1) alpha *= nlv[k + 1];
                // a one-band matvec (g_k = w_k b_k) folds into the weights:
                // pass 1 then reduces the staged rows b directly
                double wk = 1.0;
                if constexpr (NB == 1) {
                    const double2 w2 = coef(0, k >> 1);
                    wk = (k & 1) ? w2.y : w2.x;
                }
                ab_g[k * T + t] = make_double2(BC::FWD ? alpha * wk : 0.0, BC::BWD ? beta * wk : 0.0);
            }
        }
        return;
    }

    const int sw_me = swz_row<BC::SWB>(t), sw_prev = swz_row<BC::SWB>(t - 1), sw_next = swz_row<BC::SWB>(t + 1);
    const int swo_me = swz_row<BC::SWBO>(t);
    auto unit_off = [&](int u, int ch, int sw) -> uint32_t {
        return (uint32_t)((H > 1 ? (u / IB) * T : 0) + ch) * ROWB + (((u % IB) ^ sw) << 4);
    };
    const bool win_partial = io.iz0 > 0 || io.iz1 < io.M;
    // Single pass, M not a multiple of R: the tensor maps hold the first
    // Mfull rows; the thread whose chunk starts at Mfull (the tail chunk,
    // outside the maps: zero-filled by the loads, dropped by the stores)
    // moves its rows between global memory and its staged units itself.
    const int64_t Mfull = (io.M / R) * R;
    // Single pass on rows no tensor map can describe (a stride or offset
    // that is not a multiple of 16 bytes, e.g. an odd M at stride M): every
    // thread reads its rows and halo rows from global memory and writes its
    // results with plain stores; no staging, no TMA.
    const bool plain = PASS == 4 && io.plain != 0;
    const bool tail_thread = PASS == 4 && !plain && Mfull < io.M && s_glob == Mfull;
    auto in_row = [&](int64_t y, int64_t row) -> double {  // input row of system y as data (0 outside)
        if (row < 0 || row >= io.M || row < io.iz0 || row >= io.iz1) return 0.0;
        return io.in[io.in_off + y * io.in_stride + row];
    };
    const int64_t nsys = io.nsys;
    // systems in flight over the grid (passes 1 and 2: over the CTA's range)
    const int64_t per = (PASS == 1 || PASS == 2) ? (int64_t)C::G : (int64_t)(gridDim.x / (unsigned)NS) * C::G;
    int64_t sys = (int64_t)(blockIdx.x / (unsigned)NS) * C::G + grp;
    int chunk0 = c * T;

    auto issue_load = [&](unsigned char* b, uint32_t bar, int64_t y) {
        mbar_arrive_expect_tx(bar, (uint32_t)(H * 32 * ROWB));
#pragma unroll
        for (int h = 0; h < H; ++h)
            tma_load_3d(smem_u32(b + (size_t)(h * T + 32 * wg) * ROWB), &tm_in, h * IB * 2, chunk0 + 32 * wg, (int)y,
                        bar);
    };
    auto issue_store = [&](unsigned char* b, int64_t y) {
#pragma unroll
        for (int h = 0; h < BC::HO; ++h)
            tma_store_3d(&tm_out, h * IBO * 2, chunk0 + 32 * wg, (int)y,
                         smem_u32(b + (size_t)(h * T + 32 * wg) * ROWBO));
        bulk_commit();
    };


    if constexpr (PASS == 4) {
        // Pipelined single pass.  Iteration k prefetches system k+1, runs
        // phase A of system k (the slice solved with zero carries, its
        // offsets published, the result x0 staged in place of the input) and
        // phase B of system k-1 (once every slice of it has published: the
        // carries composed, their responses added, the result stored).  The
        // wait for a system's flags therefore trails its publication by a
        // whole system of work.  Three buffers per group: A's, B's and the
        // prefetch's, which reuses the buffer stored from two iterations ago.
        const int64_t sys0 = sys;
        const int64_t nk = sys0 < nsys ? (nsys - sys0 + per - 1) / per : 0;  // this group's systems
        auto bufp = [&](int64_t k) -> unsigned char* { return buf0 + (size_t)(k % 3) * BC::BUF; };
        auto barp = [&](int64_t k) -> uint32_t { return smem_u32(&bars[k % 3]); };
        auto parity = [&](int64_t k) -> uint32_t { return (uint32_t)((k / 3) & 1); };
        auto sys_of = [&](int64_t k) -> int64_t { return sys0 + k * per; };
        auto recf = [&](int64_t y, int f) -> double& { return red[((size_t)c * kLgRed + f) * nsys + y]; };
        auto stage_off = [&](int u) -> uint32_t { return unit_off(u, t, sw_me); };  // this thread's units
        constexpr bool COUPLED = BC::FWD || BC::BWD || KL > 0 || KU > 0;
        const bool tail_slice = !plain && Mfull < io.M && s0 + C::S > Mfull;
        // the halo rows of the first and last threads, loaded a system ahead
        // beside the TMA load (they are used, and so read, before the slice
        // publishes that system: no neighbour has stored it yet)
        auto halo = [&](int64_t kk, double (&h)[4]) {
            if (kk >= nk) return;
            const int64_t y = sys_of(kk);
            if constexpr (KL > 0) {
                if (t == 0) {
                    h[0] = in_row(y, s0 - 2);
                    h[1] = in_row(y, s0 - 1);
                }
            }
            if constexpr (KU > 0) {
                if (t == T - 1) {
                    h[2] = in_row(y, s0 + C::S);
                    h[3] = in_row(y, s0 + C::S + 1);
                }
            }
        };
        double hc[4] = {0.0, 0.0, 0.0, 0.0}, hn[4] = {0.0, 0.0, 0.0, 0.0};
        if (!plain) halo(0, hc);
        if (!plain && nk > 0 && lane == 0) issue_load(bufp(0), barp(0), sys_of(0));
        for (int64_t k = 0; k <= nk; ++k) {
            const bool prefetch = !plain && k + 1 < nk;
            if (prefetch) halo(k + 1, hn);
            if (prefetch && lane == 0) {
                bulk_wait_read_all();  // the store from this buffer (system k-2) has read it
                issue_load(bufp(k + 1), barp(k + 1), sys_of(k + 1));
            }
            bool ok = true;
            if (k < nk) {
                // ---- phase A of system k
                const int64_t y = sys_of(k);
                unsigned char* cur = bufp(k);
                ok = plain || mbar_wait_bounded(barp(k), parity(k));
                ok = group_and(g.bar_id, g.nthr, ok);
                if (ok) {
                    if (tail_slice) {  // the partial last chunk, outside the TMA boxes
                        if (tail_thread) {
#pragma unroll
                            for (int j = 0; j < R; ++j) {
                                const int64_t row = Mfull + j;
                                const double v = (row < io.M) ? io.in[io.in_off + y * io.in_stride + row] : 0.0;
                                reinterpret_cast<double*>(cur + stage_off(j >> 1))[j & 1] = v;
                            }
                        }
                        if (W > 1) group_bar(g.bar_id, g.nthr);
                        else __syncwarp();
                    }
                    double x[R + KL + KU];
                    if (plain) {
#pragma unroll
                        for (int i = 0; i < R + KL + KU; ++i) x[i] = in_row(y, s_glob - KL + i);
                    } else {
#pragma unroll
                        for (int u = 0; u < U; ++u) {
                            const double2 v = *reinterpret_cast<const double2*>(cur + stage_off(u));
                            x[KL + 2 * u] = v.x;
                            x[KL + 2 * u + 1] = v.y;
                        }
                        if constexpr (KL > 0) {
                            double2 pv;
                            if (t > 0) pv = *reinterpret_cast<const double2*>(cur + unit_off(U - 1, t - 1, sw_prev));
                            else pv = make_double2(hc[0], hc[1]);
                            x[KL - 1] = pv.y;
                            if constexpr (KL > 1) x[0] = pv.x;
                        }
                        if constexpr (KU > 0) {
                            double2 nv;
                            if (t < T - 1) nv = *reinterpret_cast<const double2*>(cur + unit_off(0, t + 1, sw_next));
                            else nv = make_double2(hc[2], hc[3]);
                            x[KL + R] = nv.x;
                            if constexpr (KU > 1) x[KL + R + 1] = nv.y;
                        }
                        if (win_partial) {
#pragma unroll
                            for (int i = 0; i < R + KL + KU; ++i) {
                                const int64_t row = s_glob - KL + i;
                                if (row < io.iz0 || row >= io.iz1) x[i] = 0.0;
                            }
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
                            double acc = (e ? wc[0].y : wc[0].x) * x[j];
#pragma unroll
                            for (int q = 1; q < NB; ++q) acc = __fma_rn(e ? wc[q].y : wc[q].x, x[j + q], acc);
                            x[j] = acc;
                        }
                    }
                    double Bf = 0.0, Bb0 = 0.0;
                    if constexpr (BC::FWD || BC::BWD)
                        lg_solve<C>(g, coef, Af, Ab, x,
                                    [&](double, double Bt) {
                                        Bf = Bt;
                                        return 0.0;
                                    },
                                    [&](double, double Bt) {
                                        Bb0 = Bt;
                                        return 0.0;
                                    });
                    if constexpr (COUPLED) {
                        if (t == 0) {
                            recf(y, kLgRedBf) = Bf;
                            recf(y, kLgRedBb) = Bb0;
                            st_release_u32(flags + (size_t)c * nsys + y, epoch);
                        }
                    }
                    // every thread has read its rows (the solve's scans are
                    // group barriers; without a solve, wait): stage x0
                    if constexpr (!(BC::FWD || BC::BWD)) {
                        if (W > 1) group_bar(g.bar_id, g.nthr);
                    }
                    __syncwarp();
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        *reinterpret_cast<double2*>(cur + stage_off(u)) = make_double2(x[2 * u], x[2 * u + 1]);
                }
            }
            if (ok && k >= 1) {
                // ---- phase B of system k-1
                const int64_t y = sys_of(k - 1);
                unsigned char* cur = bufp(k - 1);
                double Xin = 0.0, Yin = 0.0;
                if constexpr (COUPLED) {
                    bool ok2 = true;
                    if (wg == 0) {
                        const long long t0 = clock64();
                        for (int cc = lane; cc < NS && ok2; cc += 32)
                            while (ld_acquire_u32(flags + (size_t)cc * nsys + y) != epoch) {
                                if (clock64() - t0 > kLgWaitCycles) {
                                    ok2 = false;
                                    break;
                                }
                                __nanosleep(32);
                            }
                        ok2 = __all_sync(FULL, ok2) != 0;
                        if (ok2 && (BC::FWD || BC::BWD)) {
                            lg_compose<BC::FWD, BC::BWD>(lane, c, NS, nsys, y, red, cst_s, Xin, Yin);
                            if (lane == 0) {
                                g.warp_area(0)[16] = Xin;
                                g.warp_area(0)[17] = Yin;
                            }
                        }
                    }
                    if (W > 1) {
                        ok2 = group_and(g.bar_id, g.nthr, ok2);
                        if (wg != 0) {
                            Xin = g.warp_area(0)[16];
                            Yin = g.warp_area(0)[17];
                        }
                        group_bar(g.bar_id, g.nthr);  // the slot is read before the next system rewrites it
                    }
                    ok = ok2;
                }
                if (ok) {
                    double x[R];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const double2 v = *reinterpret_cast<const double2*>(cur + stage_off(u));
                        x[2 * u] = v.x;
                        x[2 * u + 1] = v.y;
                    }
                    if constexpr (BC::FWD || BC::BWD) {
#pragma unroll
                        for (int j = 0; j < R; ++j) {
                            const double2 pg = ab_s[j * T + t];
                            x[j] = __fma_rn(Xin, pg.x, __fma_rn(Yin, pg.y, x[j]));
                        }
                    }
                    if (C::SV != SV_NONE && s_glob == 0) x[0] = op.scaleC * x[0];
                    if (plain || tail_thread) {  // plain stores (the TMA store drops the tail chunk)
                        const int64_t r0 = plain ? s_glob : Mfull;
#pragma unroll
                        for (int j = 0; j < R; ++j) {
                            const int64_t row = r0 + j;
                            if (row < io.M && row >= io.oz0 && row < io.oz1)
                                io.out[io.out_off + y * io.out_stride + row] = x[j];
                        }
                    }
                    if (!plain) {
#pragma unroll
                        for (int u = 0; u < U; ++u)
                            *reinterpret_cast<double2*>(cur + stage_off(u)) = make_double2(x[2 * u], x[2 * u + 1]);
                        fence_proxy_async();
                        __syncwarp();
                        if (lane == 0) issue_store(cur, y);
                    }
                }
            }
            if (!ok) {
                if (t == 0) atomicOr(&g_stream_status, kStatusWaitTimeout);
                // the prefetched load completes before the CTA exits
                if (prefetch && lane == 0) mbar_wait_bounded(barp(k + 1), parity(k + 1));
                break;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) hc[i] = hn[i];
        }
        if (lane == 0) bulk_wait_all();
        return;
    }

    // The per-system scalars a pass reads from global memory -- the halo rows
    // (the input in pass 1, the records in pass 2) and pass 2's carries -- are
    // loaded a system ahead, beside the next system's TMA load, so that their
    // latency is not in the solve's path.
    struct Scal {
        double lo0, lo1, hi0, hi1, X, Y;
    };
    int64_t ylim = 0;  // end of the current segment's systems
    auto fetch = [&](int64_t y) -> Scal {
        Scal r{0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (y >= ylim) return r;
        auto rv = [&](int k) -> double { return red[((size_t)c * kLgRed + k) * nsys + y]; };
        if constexpr (KL > 0) {
            if (t == 0) {
                r.lo0 = PASS == 1 ? in_row(y, s0 - 2) : rv(kLgRedLo);
                r.lo1 = PASS == 1 ? in_row(y, s0 - 1) : rv(kLgRedLo + 1);
            }
        }
        if constexpr (KU > 0) {
            if (t == T - 1) {
                r.hi0 = PASS == 1 ? in_row(y, s0 + C::S) : rv(kLgRedHi);
                r.hi1 = PASS == 1 ? in_row(y, s0 + C::S + 1) : rv(kLgRedHi + 1);
            }
        }
        if constexpr (PASS == 2) {
            if constexpr (BC::FWD) r.X = rv(kLgRedX);
            if constexpr (BC::BWD) r.Y = rv(kLgRedY);
        }
        return r;
    };
    // The CTA's range in segments of one slice each; at a slice change every
    // group has finished with the old table (no load of this CTA is in
    // flight then: the last item of a segment prefetches nothing).
    int kk = 0;  // items this group has run: its buffer and barrier phase
    bool stop = false;
    for (int64_t seg = it_beg; seg < it_end;) {
        const int cs = (int)(seg / nsys);
        const int64_t seg_end = it_end < (int64_t)(cs + 1) * nsys ? it_end : (int64_t)(cs + 1) * nsys;
        if (cs != c) {
            __syncthreads();
            c = cs;
            s0 = (int64_t)c * C::S;
            s_glob = s0 + (int64_t)t * R;
            chunk0 = c * T;
            load_slice();
            __syncthreads();
            chunk_mults();
        }
        sys = seg - (int64_t)cs * nsys + grp;
        ylim = seg_end - (int64_t)cs * nsys;
        seg = seg_end;
        if (stop) continue;
        // M not a multiple of R: the tensor maps hold the first Mfull rows,
        // and the thread whose chunk starts at Mfull (in this segment's
        // slice, if at all) copies its rows of each system into a slot of its
        // own by cp.async, beside the system's TMA load, stages them after the
        // load's wait, and stores its results with plain stores
        const bool tail_thr = Mfull < io.M && s_glob == Mfull;
        const bool tail_slice = Mfull < io.M && s0 + C::S > Mfull;
        auto tail_copy = [&](int slot, int64_t y) {
            const double* src = io.in + io.in_off + y * io.in_stride + Mfull;
            double* dst = tail_s + slot * R;
            const int64_t have = io.M - Mfull;  // rows present, 1 .. R-1
#pragma unroll
            for (int j = 0; j < R; j += 2) {
                const int64_t nb = have - j <= 0 ? 0 : (have - j >= 2 ? 16 : 8);
                cp_async16n(dst + j, nb ? src + j : src, (int)nb);
            }
            cp_async_commit();
        };
        Scal sc = fetch(sys), scn;
        if (sys < ylim && tail_thr) tail_copy(kk & 1, sys);
        if (sys < ylim && lane == 0) {
            if (PASS == 2) bulk_wait_read_all();  // the store from this buffer (two items ago) has read it
            issue_load((kk & 1) ? buf1 : buf0, (kk & 1) ? bar1 : bar0, sys);
        }
        for (; sys < ylim; ++kk, sys += per, sc = scn) {
            unsigned char* cur = (kk & 1) ? buf1 : buf0;
            unsigned char* nxt = (kk & 1) ? buf0 : buf1;
            const bool more = sys + per < ylim;
            scn = fetch(sys + per);
            bool ok = mbar_wait_bounded((kk & 1) ? bar1 : bar0, (uint32_t)((kk >> 1) & 1));
            ok = group_and(g.bar_id, g.nthr, ok);
            if (!ok) {
                if (t == 0) atomicOr(&g_stream_status, kStatusWaitTimeout);
                stop = true;
                break;
            }
            // field k of this (system, slice) record
            auto rec = [&](int k) -> double& { return red[((size_t)c * kLgRed + k) * nsys + sys]; };
            // the partial chunk's rows into the staged units (the TMA filled
            // them with zeros); its neighbours read its first unit as their
            // halo, after the group barrier
            if (tail_slice) {
                if (tail_thr) {
                    cp_async_wait<0>();
                    const double* src = tail_s + (kk & 1) * R;
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        *reinterpret_cast<double2*>(cur + unit_off(u, t, sw_me)) =
                            *reinterpret_cast<const double2*>(src + 2 * u);
                }
                if (W > 1) group_bar(g.bar_id, g.nthr);
                else __syncwarp();
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
                } else {
                    pv = make_double2(sc.lo0, sc.lo1);
                    if (PASS == 1) {
                        rec(kLgRedLo) = pv.x;
                        rec(kLgRedLo + 1) = pv.y;
                    }
                }
                be[KL - 1] = pv.y;
                if constexpr (KL > 1) be[0] = pv.x;
            }
            if constexpr (KU > 0) {
                double2 nv = make_double2(0.0, 0.0);
                if (t < T - 1) {
                    nv = *reinterpret_cast<const double2*>(cur + unit_off(0, t + 1, sw_next));
                } else {
                    nv = make_double2(sc.hi0, sc.hi1);
                    if (PASS == 1) {
                        rec(kLgRedHi) = nv.x;
                        rec(kLgRedHi + 1) = nv.y;
                    }
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
            // the matvec (pass 1 with a one-band matvec: folded into its
            // weights by the table pass)
            if constexpr (!(PASS == 1 && NB == 1)) {
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
            }
            double (&x)[R + KL + KU] = be;
            // `nxt` was read in the previous iteration by every warp of the group
            // (all of them have passed this iteration's group_and since) and, in
            // pass 2, stored from: once this warp's stores have read it, it takes
            // the next system
            if (more && tail_thr) tail_copy((kk + 1) & 1, sys + per);
            if (more && lane == 0) {
                if (PASS == 2) bulk_wait_read_all();
                issue_load(nxt, (kk & 1) ? bar0 : bar1, sys + per);
            }
            if constexpr (PASS == 1) {
                if constexpr (BC::FWD || BC::BWD) {
                    // Bf = sum alpha g, Bb0 = sum beta g over the slice
                    double sa = 0.0, sb = 0.0;
#pragma unroll
                    for (int j = 0; j < R; ++j) {
                        const double2 w = ab_s[j * T + t];
                        sa = __fma_rn(w.x, x[j], sa);
                        sb = __fma_rn(w.y, x[j], sb);
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        sa += __shfl_xor_sync(FULL, sa, o);
                        sb += __shfl_xor_sync(FULL, sb, o);
                    }
                    if (W > 1) {
                        double* my = g.warp_area(wg) + 16;
                        if (lane == 0) {
                            my[0] = sa;
                            my[1] = sb;
                        }
                        group_bar(g.bar_id, g.nthr);
                        if (t == 0) {
                            sa = 0.0;
                            sb = 0.0;
                            for (int w = 0; w < W; ++w) {
                                sa += g.warp_area(w)[16];
                                sb += g.warp_area(w)[17];
                            }
                        }
                    }
                    if (t == 0) {
                        if constexpr (BC::FWD) rec(kLgRedBf) = sa;
                        if constexpr (BC::BWD) rec(kLgRedBb) = sb;
                    }
                }
                continue;
            } else {
                // carries of this system's slice, from the carry kernel
                const double Xc = sc.X, Yc = sc.Y;
                lg_solve<C>(g, coef, Af, Ab, x, [&](double, double) { return Xc; }, [&](double, double) { return Yc; });
            }
            if (C::SV != SV_NONE && s_glob == 0) x[0] = op.scaleC * x[0];
            __syncwarp();
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int h = u / IBO, uu = u % IBO;
                *reinterpret_cast<double2*>(cur + (size_t)(h * T + t) * ROWBO + ((uu ^ swo_me) << 4)) =
                    make_double2(x[2 * u], x[2 * u + 1]);
            }
            if (tail_thr) {  // plain stores (the TMA store drops the tail chunk)
#pragma unroll
                for (int j = 0; j < R; ++j) {
                    const int64_t row = Mfull + j;
                    if (row < io.M && row >= io.oz0 && row < io.oz1) io.out[io.out_off + sys * io.out_stride + row] = x[j];
                }
            }
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) issue_store(cur, sys);
        }
    }
    cp_async_wait<0>();  // a partial chunk's copy of an item a wait gave up on
    if (lane == 0) bulk_wait_all();
}

}  // namespace pfb
