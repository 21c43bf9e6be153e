// jw_stream.cuh -- the streaming JW-step kernel: whole systems staged by TMA.
//
// Same operator as jw_step_kernel (x = diag(s) M^{-1} V A b, x[0] *= scaleC;
// PfSolve/pfSolve_CodeGen/pfSolve_KernelsLevel2/pfSolve_JonesWorland.h:38-408),
// organised for throughput on long runs of systems that share one matrix:
//
//  * One CTA per SM, G groups of W warps; a group owns one system at a time,
//    thread t of the group owns the R consecutive rows [R t, R t + R).
//  * Right-hand sides move global -> shared with TMA tensor loads
//    (cp.async.bulk.tensor, 3-D view {row-in-chunk, chunk, system}) into a
//    swizzled layout in which both the TMA write and the per-thread chunk read
//    are free of bank conflicts; results go back with TMA tensor stores from
//    the same buffer.  Two buffers per group: the next system's load is in
//    flight while the current one is solved.  One elected lane per warp
//    issues all copies, so moving data costs a handful of instructions per
//    system instead of one per element.
//  * The coefficients (V A folded with the LU scaling, -l, -h, Scale factors)
//    are built once per CTA, by all its threads, into a shared table read with
//    16-byte loads; the products of -l and -h over each chunk (the scan
//    multipliers) are formed once per thread.
//  * The chunk-boundary couplings are resolved with the affine scans of the
//    group kernel (warp shuffles, then shared memory across warps).
//  * Completion waits are bounded: a wait that exceeds its limit records
//    kStatusWaitTimeout in the device status word and the CTA stops.
//  * Storage is FP64 or FP32 (PREC_F32, PREC_F64_F32MEM); a 16-byte unit of a
//    staged plane holds 2 or 4 rows.  The staging buffer is warp-major: the
//    boxes of warp w's 32 chunks (every plane and swizzle row) come before
//    warp w+1's, for the input and for the output layout, so each warp's
//    input and output bytes coincide and the warp's own bulk-copy waits order
//    its next load after its last store.
#pragma once
#include <cuda.h>

#include "jw_kernel.cuh"

namespace pfb {

// Component e (0..3, a compile-time index after unrolling) of a float4.
__device__ __forceinline__ float f4_at(const float4& v, int e)
{
    return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w));
}

constexpr unsigned kStatusWaitTimeout = 1u;
static __device__ unsigned int g_stream_status;

// PRODS_: 0 leaves out the chunk-product planes (the long-system kernels use
// this layout for their slice tables and form their products themselves).
template <int R_, int W_, int KL_, int KU_, int SV_, int LIN_, int LOUT_, bool SCALE_, int PREC_ = PREC_F64,
          int ALT_ = 0, int PRODS_ = 1>
struct StCfg {
    static constexpr int R = R_, W = W_, KL = KL_, KU = KU_, SV = SV_, LIN = LIN_, LOUT = LOUT_;
    static constexpr bool SCALE = SCALE_;
    // ALT stride-2 mode (pfSolve_TridiagonalSolve.h:1319-1330, 1622-1644): the
    // even rows and the odd rows of a staged row set are two systems.  A
    // 16-byte unit holds rows 2u and 2u + 1, one row of each system with the
    // same index in it, and a row's neighbours in its system are S = 2 rows
    // away; the staged halo is S KL rows before and S KU rows after a chunk.
    static constexpr bool ALT = ALT_ != 0;
    static constexpr int S = ALT ? 2 : 1;
    static constexpr int KLP = S * KL_, KUP = S * KU_;
    static constexpr bool CPLX = (LIN != LAY_REAL);
    static constexpr bool F32MEM = prec_f32_storage(PREC_);  // FP32 storage
    static constexpr bool F32 = (PREC_ == PREC_F32);          // FP32 arithmetic
    using Sto = typename std::conditional<F32MEM, float, double>::type;  // storage scalar
    using MS = typename std::conditional<F32, float, double>::type;     // arithmetic scalar
    using CT = MS;                                                       // coefficient table scalar
    using CT2 = typename Vec2Of<CT>::type;                              // one table entry: a row pair
    static constexpr int ES = (int)sizeof(Sto);
    using V = typename std::conditional<CPLX, typename Vec2Of<MS>::type, MS>::type;
    using VF = typename Lower<V>::type;
    static constexpr int T = 32 * W;  // chunks (threads) per group
    static constexpr int NB = KL + KU + 1;
    static constexpr bool FWD = (SV == SV_LOWER || SV == SV_TRI);
    static constexpr bool BWD = (SV == SV_UPPER || SV == SV_TRI);
    static constexpr bool MIXED = (PREC_ == PREC_MIXED) && (SV != SV_NONE);
    // Coefficient table planes, each one CT2 per (row pair, thread).
    // FP64 / FP32: NB weights (scaled by the LU pivots), -l, -h, Scale factor.
    // Mixed: NB weights (unscaled), the solve's sub- and super-diagonal in FP64
    // (residual), FP32 packs {m, m', -l, -l'} and {-h, -h', 0, 0}, Scale factor.
    // FP32 arithmetic, 16 or 32 rows per thread (QUAD): one float4 per (row
    // quad, thread), and two more planes, the products of -l over the chunk's
    // rows up to each row and of -h from each row on, so that a system's
    // coupling terms cost one FMA a row.  (At 8 rows per thread the extra
    // table loads measured slower than forming the products per system.)
    static constexpr bool QUAD = F32 && R >= 16 && PRODS_;
    // FP64 storage and arithmetic, 16 or 32 rows per thread (PROD): the same
    // two planes of chunk products, as row pairs (measured: config 3, N = 512,
    // 0.197 -> 0.179 ms; on FP32 storage with FP64 arithmetic it measured
    // slower at N = 512, so those variants keep the per-system products).
    static constexpr bool PROD = PREC_ == PREC_F64 && !ALT_ && R >= 16 && PRODS_;
    static constexpr bool PRODS = QUAD || PROD;
    static constexpr int P_NL = NB, P_NH = NB + (FWD ? 1 : 0);  // FP64 / FP32 path
    static constexpr int P_AL = NB, P_CU = NB + (FWD ? 1 : 0);  // mixed path
    static constexpr int P_F1 = P_CU + (BWD ? 1 : 0), P_F2 = P_F1 + 1;
    static constexpr int P_PL = P_NH + (BWD ? 1 : 0), P_PH = P_PL + ((PRODS && FWD) ? 1 : 0);  // QUAD / PROD
    static constexpr int P_SC = MIXED ? P_F2 + (BWD ? 1 : 0) : (PRODS ? P_PH + (BWD ? 1 : 0) : P_NH + (BWD ? 1 : 0));
    static constexpr int NPL = P_SC + (SCALE ? 1 : 0);
    static constexpr int U4 = R / 4;  // QUAD: row quads per chunk
    // Table: U row pairs per chunk.
    static constexpr int U = R / 2;
    // Input: NPIN planes of ES-byte rows; a 16-byte unit holds EPU rows, a
    // chunk UD units per plane, stored as H swizzle rows of IB units (TMA box
    // inner extent).
    static constexpr int NPIN = CPLX ? 2 : 1;
    static constexpr int EPU = 16 / ES;
    static constexpr int UD = R / EPU;
    static constexpr int IB = UD < 8 ? UD : 8;
    static constexpr int H = UD / IB;
    static constexpr int SWB = Log2<IB>::v;
    // Output: packed complex (2 ES-byte rows) or planes of ES-byte rows; a
    // 16-byte unit holds EPUO rows.
    static constexpr bool OPK = (LOUT == LAY_PACKED);
    static constexpr int NPOUT = OPK ? 1 : (LOUT == LAY_XXII ? 2 : 1);
    static constexpr int EPUO = OPK ? 8 / ES : EPU;
    static constexpr int UO = R / EPUO;
    static constexpr int IBO = UO < 8 ? UO : 8;
    static constexpr int HO = UO / IBO;
    static constexpr int SWBO = Log2<IBO>::v;
    static constexpr size_t BUF = (size_t)T * R * ES * (CPLX ? 2 : 1);  // bytes of one system
    // Table rows of T 16-byte units, padded by one unit: the prologue's
    // writes (consecutive threads on consecutive row pairs of one chunk) then
    // fall on different banks; the loop's reads (consecutive threads on
    // consecutive units of one row) are conflict-free either way.
    static constexpr int TP = (W <= 2) ? T + 1 : T;  // 4-warp groups: no room to spare at N = 4096
    static constexpr size_t TBL = (size_t)NPL * U * TP * sizeof(CT2);
    // Bytes per chunk of the input and of the output layout (equal: a system
    // is staged in place); with the warp-major layout, warp w's input and
    // output bytes are then the same range.
    static constexpr int ROWB = IB * 16, ROWBO = IBO * 16;
    static_assert(NPIN * H * ROWB == NPOUT * HO * ROWBO, "in-place staging");
    // Registers held by the right-hand-side data (mixed: x and the FP32
    // correction; g waits in shared memory); the launch bound leaves the compiler room for them:
    // 512 threads cap at 128 registers, 384 at 170, 256 at 255.  Complex
    // variants stay at 256 (measured faster than 384 on the config 2 chain).
    static constexpr int kDataRegs =
        (R + KLP + KUP) * (CPLX ? 2 : 1) * (F32 ? 1 : 2) + (MIXED ? R * (CPLX ? 2 : 1) : 0);
    static constexpr int kMaxThreads =
        (kDataRegs >= 96 || (CPLX && kDataRegs >= 64)) ? 256 : (kDataRegs >= 64 ? 384 : 512);
    static_assert(R % 2 == 0 && R >= 4 && R <= 32, "rows per thread");
    static_assert(!QUAD || R % 4 == 0, "FP32: whole row quads per chunk");
    static_assert(KLP <= 2 && KUP <= 2, "halo of at most two rows");
    static_assert(!ALT || (!CPLX && !MIXED && !SCALE && !F32MEM), "ALT: real FP64 systems without a Scale epilogue");
    static_assert(!MIXED || !F32MEM, "mixed precision: FP64 storage");
    static_assert(CPLX ? (LOUT != LAY_REAL) : (LOUT == LAY_REAL), "layout pair");
};

// NB: staging buffers per group (2..kStMaxBuffers).
template <class C>
__host__ __device__ constexpr size_t st_fixed_bytes(int G, int NB)
{
    return C::TBL + (size_t)G * C::W * kScratchPerWarp * sizeof(double) + (size_t)G * NB * sizeof(uint64_t);
}

// Dynamic shared memory: table | scratch | mbarriers | (align 1024) | buffers.
template <class C>
__host__ __device__ constexpr size_t st_smem_bytes(int G, int NB)
{
    return st_fixed_bytes<C>(G, NB) + 1024 + (size_t)G * NB * C::BUF;
}

// ---- TMA, mbarrier and bulk-group primitives (PTX).
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for phase `parity` of `bar`, giving up after about two seconds.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > 4000000000LL) return false;
    return true;
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z, uint32_t src)
{
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(z), "r"(src)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// AND of `pred` over the `nthreads` threads of named barrier `id`.
__device__ __forceinline__ bool group_and(int id, int nthreads, bool pred)
{
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

// XOR pattern of the TMA swizzle for a row of 2^B 16-byte units: unit u of
// swizzle row t lands at unit u ^ ((t >> (3 - B)) & (2^B - 1)).
template <int B>
__device__ __forceinline__ int swz_row(int t)
{
    if constexpr (B == 0) return 0;
    else return (t >> (3 - B)) & ((1 << B) - 1);
}

// ---- Coefficient table, built once per CTA by all of its threads.
// Plane p, row i = R*tt + j (tt: thread of a group) is the double at
// [((p*U + j/2)*T + tt)*2 + (j&1)]: thread tt reads rows 2u, 2u+1 of a plane
// as one 16-byte word, lanes on consecutive words.
template <class C>
__device__ void st_prologue_system(const JwOperator& op, int h, typename C::CT* table, GroupCtx& g)
{
    constexpr int R = C::R, T = C::T, U = C::U, NB = C::NB;
    const int64_t M = op.M;
    const int rows = T * R / C::S;
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int Rp = (rows + nthr - 1) / nthr;
    const int64_t s = (int64_t)tid * Rp;
    double dprev = 1.0;
    if constexpr (C::SV == SV_TRI) {
        // Moebius product of this thread's rows, then the CTA-wide scan gives
        // the pivot entering them (same recurrence as jw_prologue).
        double a = 1, b = 0, c = 0, d = 1;
        for (int j = 0; j < Rp; ++j) {
            const int64_t i = s + j;
            double ac = 0.0;
            if (i >= 1 && i < M) ac = band(op, op.off_sl, i) * band(op, op.off_su, i - 1);
            const double na = a - ac * c, nb = b - ac * d;
            c = a;
            d = b;
            a = na;
            b = nb;
            renorm2x2(a, b, c, d);
        }
        group_matrix_scan(g, a, b, c, d);
        dprev = (s == 0) ? 1.0 : a / c;
    }
    for (int j = 0; j < Rp; ++j) {
        const int64_t i = s + j;
        if (i >= rows) break;
        double w[NB];
        double nl = 0.0, nh = 0.0, sc = 0.0, m = 1.0, al = 0.0, cu = 0.0;
        if (i < M) {
            jw_row_weights<C::KL, NB>(op, i, w);
            if constexpr (C::SV == SV_TRI) {
                const double ai = (i >= 1) ? band(op, op.off_sl, i) : 0.0;
                const double ci = (i < M - 1) ? band(op, op.off_su, i) : 0.0;
                const double ac = (i >= 1) ? ai * band(op, op.off_su, i - 1) : 0.0;
                const double dp = (i == 0) ? 1.0 : 1.0 - ac / dprev;
                m = 1.0 / dp;
                dprev = dp;
                nl = -(ai * m);
                nh = -(ci * m);
                al = ai;
                cu = ci;
            } else if constexpr (C::SV == SV_LOWER) {
                al = (i >= 1) ? band(op, op.off_sl, i) : 0.0;
                nl = -al;
            } else if constexpr (C::SV == SV_UPPER) {
                cu = (i < M - 1) ? band(op, op.off_su, i) : 0.0;
                nh = -cu;
            }
            if constexpr (!C::MIXED) {
#pragma unroll
                for (int k = 0; k < NB; ++k) w[k] *= m;
            }
            if constexpr (C::SCALE) sc = scale_factor(op.scale_kind, i, op.lshift, op.scale_s);
        } else {
#pragma unroll
            for (int k = 0; k < NB; ++k) w[k] = 0.0;
        }
        const int64_t si = C::S * i + h;  // staged row
        const int tt = (int)(si / R), jj = (int)(si % R);
        auto put = [&](int p, double v) {
            table[(((size_t)p * U + (jj >> 1)) * C::TP + tt) * 2 + (jj & 1)] = (typename C::CT)v;
        };
        if constexpr (C::QUAD) {  // float4 per (row quad, thread)
            const int q4 = jj >> 2, e4 = jj & 3;
            auto putq = [&](int p, double v) {
                reinterpret_cast<float*>(table)[(((size_t)p * C::U4 + q4) * C::TP + tt) * 4 + e4] = (float)v;
            };
#pragma unroll
            for (int k = 0; k < NB; ++k) putq(k, w[k]);
            if constexpr (C::FWD) putq(C::P_NL, nl);
            if constexpr (C::BWD) putq(C::P_NH, nh);
            if constexpr (C::SCALE) putq(C::P_SC, sc);
            continue;
        }
        auto put32 = [&](int p, int k, double v) {
            reinterpret_cast<float*>(table)[(((size_t)p * U + (jj >> 1)) * C::TP + tt) * 4 + k + (jj & 1)] = (float)v;
        };
#pragma unroll
        for (int k = 0; k < NB; ++k) put(k, w[k]);
        if constexpr (C::MIXED) {
            if constexpr (C::FWD) put(C::P_AL, al);
            if constexpr (C::BWD) put(C::P_CU, cu);
            put32(C::P_F1, 0, m);
            put32(C::P_F1, 2, nl);
            if constexpr (C::BWD) {
                put32(C::P_F2, 0, nh);
                put32(C::P_F2, 2, 0.0);
            }
        } else {
            if constexpr (C::FWD) put(C::P_NL, nl);
            if constexpr (C::BWD) put(C::P_NH, nh);
        }
        if constexpr (C::SCALE) put(C::P_SC, sc);
    }
}

// Coefficient table of the staged system(s), built by all threads of the CTA.
// ALT: system h is the parity-h rows, with its own row count and band
// positions (the group kernel's per-parity operator, jw_step_kernel).
template <class C>
__device__ void st_prologue(const JwOperator& op, typename C::CT* table, double* scratch_all)
{
    GroupCtx g;
    g.lane = threadIdx.x & 31;
    g.wg = threadIdx.x >> 5;
    g.W = blockDim.x >> 5;
    g.nthr = blockDim.x;
    g.bar_id = 1;
    g.seq = 0;
    g.scratch = scratch_all;
    if constexpr (!C::ALT) {
        st_prologue_system<C>(op, 0, table, g);
        if constexpr (C::PROD && (C::FWD || C::BWD)) {
            // one thread per chunk: the products of -l up to each row and of
            // -h from each row on, in the order the solve used to form them
            __syncthreads();
            auto at = [&](int p, int j, int tt) -> double& {
                return table[(((size_t)p * C::U + (j >> 1)) * C::TP + tt) * 2 + (j & 1)];
            };
            for (int tt = threadIdx.x; tt < C::T; tt += blockDim.x) {
                if constexpr (C::FWD) {
                    double pr = 1.0;
                    for (int j = 0; j < C::R; ++j) {
                        pr = at(C::P_NL, j, tt) * pr;
                        at(C::P_PL, j, tt) = pr;
                    }
                }
                if constexpr (C::BWD) {
                    double pr = 1.0;
                    for (int j = C::R - 1; j >= 0; --j) {
                        pr = at(C::P_NH, j, tt) * pr;
                        at(C::P_PH, j, tt) = pr;
                    }
                }
            }
        }
        if constexpr (C::QUAD && (C::FWD || C::BWD)) {
            // one thread per chunk: the products of -l up to each row and of
            // -h from each row on, in the order the solve used to form them
            __syncthreads();
            float* tf = reinterpret_cast<float*>(table);
            auto at = [&](int p, int j, int tt) -> float& {
                return tf[(((size_t)p * C::U4 + (j >> 2)) * C::TP + tt) * 4 + (j & 3)];
            };
            for (int tt = threadIdx.x; tt < C::T; tt += blockDim.x) {
                if constexpr (C::FWD) {
                    float pr = 1.0f;
                    for (int j = 0; j < C::R; ++j) {
                        pr = at(C::P_NL, j, tt) * pr;
                        at(C::P_PL, j, tt) = pr;
                    }
                }
                if constexpr (C::BWD) {
                    float pr = 1.0f;
                    for (int j = C::R - 1; j >= 0; --j) {
                        pr = at(C::P_NH, j, tt) * pr;
                        at(C::P_PH, j, tt) = pr;
                    }
                }
            }
        }
    } else {
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            JwOperator oph = op;
            oph.alt_h = h;
            oph.M = (op.M - h + 1) >> 1;
            st_prologue_system<C>(oph, h, table, g);
        }
    }
}

// ---- The kernel.
template <class C>
__global__ void __launch_bounds__(C::kMaxThreads) jw_stream_kernel(const __grid_constant__ CUtensorMap tm_in,
                                                                  const __grid_constant__ CUtensorMap tm_out,
                                                                  const JwOperator op, const JwIO io)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using V = typename C::V;
    using O = VOps<V>;
    using MS = typename C::MS;
    using CT = typename C::CT;
    using CT2 = typename C::CT2;
    constexpr int R = C::R, W = C::W, T = C::T, U = C::U, NB = C::NB, S = C::S;
    constexpr int EPU = C::EPU, UD = C::UD, UO = C::UO, ES = C::ES;
    constexpr int KL = C::KLP, KU = C::KUP;  // staged halo rows (S times the band halo)
    constexpr int IB = C::IB, H = C::H, IBO = C::IBO, HO = C::HO;
    const int G = blockDim.x / T;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = warp / W, wg = warp - grp * W;

    CT* table = reinterpret_cast<CT*>(smem_raw);
    double* scratch_all = reinterpret_cast<double*>(smem_raw + C::TBL);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + C::TBL + (size_t)G * W * kScratchPerWarp * sizeof(double));
    // NBUF staging buffers per group, used in turn: system k of the group in
    // buffer k mod NBUF, its load issued NBUF - 1 systems ahead.
    const int NBUF = (io.nbuf >= 2 && io.nbuf <= kStMaxBuffers) ? io.nbuf : 2;
    unsigned char* after = reinterpret_cast<unsigned char*>(bars + NBUF * G);
    const uint32_t pad = (1024u - (smem_u32(after) & 1023u)) & 1023u;
    unsigned char* buf_base = after + pad + (size_t)(NBUF * grp) * C::BUF;
    auto buf_at = [&](int b) -> unsigned char* { return buf_base + (size_t)b * C::BUF; };
    auto bar_at = [&](int b) -> uint32_t { return smem_u32(&bars[NBUF * grp + b]); };

    // Shared-memory byte offset of swizzle row h of plane p of chunk c, in the
    // warp-major staging layout (the boxes of warp c/32, then the next
    // warp's); unit uu (< IB) of that row is at + ((uu ^ swz(c)) << 4).
    constexpr int ROWB = C::ROWB, ROWBO = C::ROWBO;
    auto in_row = [&](int p, int h, int c) -> size_t {
        return ((size_t)(((c >> 5) * C::NPIN + p) * H + h) * 32 + (c & 31)) * ROWB;
    };
    auto out_row = [&](int p, int h, int c) -> size_t {
        return ((size_t)(((c >> 5) * C::NPOUT + p) * HO + h) * 32 + (c & 31)) * ROWBO;
    };
    const int64_t nsys = io.nsys;
    const int64_t step = (int64_t)gridDim.x * G;
    int64_t sys = (int64_t)blockIdx.x * G + grp;

    // lane 0 of each warp: load / store this warp's 32 chunks of one system
    // (TMA x coordinates in storage elements: 16 / ES per 16-byte unit)
    auto issue_load = [&](unsigned char* b, uint32_t bar, int64_t y) {
        mbar_arrive_expect_tx(bar, (uint32_t)(C::NPIN * H * 32 * ROWB));
#pragma unroll
        for (int p = 0; p < C::NPIN; ++p)
#pragma unroll
            for (int h = 0; h < H; ++h)
                tma_load_3d(smem_u32(b + in_row(p, h, 32 * wg)), &tm_in, h * IB * (16 / ES), 32 * wg,
                            (int)(C::CPLX ? 2 * y + p : y), bar);
    };
    auto issue_store = [&](unsigned char* b, int64_t y) {
#pragma unroll
        for (int p = 0; p < C::NPOUT; ++p)
#pragma unroll
            for (int h = 0; h < HO; ++h)
                tma_store_3d(&tm_out, h * IBO * (16 / ES), 32 * wg, (int)(C::NPOUT == 2 ? 2 * y + p : y),
                             smem_u32(b + out_row(p, h, 32 * wg)));
        bulk_commit();
    };

    if ((int)threadIdx.x < NBUF * G) mbar_init(smem_u32(&bars[threadIdx.x]), W);
    mbar_init_fence();
    __syncthreads();  // the barriers are initialised before any copy can complete on them
    // The first system's copy does not depend on the coefficient table: it is
    // in flight while the prologue reads the bands.
    if (lane == 0)
        for (int j = 0; j < NBUF - 1 && sys + j * step < nsys; ++j) issue_load(buf_at(j), bar_at(j), sys + j * step);
    st_prologue<C>(op, table, scratch_all);
    __syncthreads();

    GroupCtx g;
    g.lane = lane;
    g.wg = wg;
    g.W = W;
    g.nthr = T;
    g.bar_id = 1 + grp;
    g.seq = 0;
    g.scratch = scratch_all + (size_t)grp * W * kScratchPerWarp;

    const int t = wg * 32 + lane;
    const int64_t s = (int64_t)t * R;
    const CT2* tb = reinterpret_cast<const CT2*>(table) + t;  // pair (p, u) at tb[(p*U + u)*TP]
    auto coef = [&](int p, int u) -> CT2 { return tb[(p * U + u) * C::TP]; };

    auto coef4 = [&](int p, int u) -> float4 { return reinterpret_cast<const float4*>(tb)[(p * U + u) * C::TP]; };
    // Mixed precision, real systems of up to 16 rows per thread: the FP32 solve
    // factors {m, -l} stay in registers for the whole kernel (every refinement
    // sweep reuses them); {-h} too for up to 8 rows per thread (at 16, the
    // 128-register bound of a 512-thread CTA leaves no room for them).
    constexpr bool kHoist = C::MIXED && !C::CPLX && U <= 8;
    constexpr bool kHoist2 = kHoist && U <= 4;
    float4 hf1[kHoist ? U : 1];
    float2 hf2[kHoist2 ? U : 1];
    if constexpr (kHoist) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            hf1[u] = coef4(C::P_F1, u);
            if constexpr (kHoist2 && C::BWD) {
                const float4 f = coef4(C::P_F2, u);
                hf2[u] = make_float2(f.x, f.y);
            } else if constexpr (kHoist2) {
                hf2[u] = make_float2(0.0f, 0.0f);
            }
        }
    }
    auto F1 = [&](int u) -> float4 {
        if constexpr (kHoist) return hf1[u];
        else return coef4(C::P_F1, u);
    };
    auto F2 = [&](int u) -> float2 {
        if constexpr (kHoist2) {
            return hf2[u];
        } else {
            const float4 f = coef4(C::P_F2, u);
            return make_float2(f.x, f.y);
        }
    };

    // Scan multipliers: products of -l and -h over this thread's chunk (in the
    // precision of the solve that uses them).
    // ALT: one multiplier per system, Af / Ab for the even rows and Af1 / Ab1
    // for the odd rows.
    CT Af = 1, Ab = 1, Af1 = 1, Ab1 = 1;
    float Af32 = 1.0f, Ab32 = 1.0f;
    // QUAD: row quad q of plane p as a float4
    auto coefq = [&](int p, int q) -> float4 {
        return reinterpret_cast<const float4*>(table)[((size_t)p * C::U4 + q) * C::TP + t];
    };
    if constexpr (C::QUAD) {
        if constexpr (C::FWD) Af = (CT)coefq(C::P_PL, C::U4 - 1).w;
        if constexpr (C::BWD) Ab = (CT)coefq(C::P_PH, 0).x;
    }
    if constexpr (C::PROD) {
        if constexpr (C::FWD) Af = coef(C::P_PL, U - 1).y;
        if constexpr (C::BWD) Ab = coef(C::P_PH, 0).x;
    }
    if constexpr (C::FWD && !C::MIXED && !C::QUAD && !C::PROD) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const CT2 c = coef(C::P_NL, u);
            if constexpr (C::ALT) {
                Af = c.x * Af;
                Af1 = c.y * Af1;
            } else {
                Af = (u == 0) ? c.x : c.x * Af;
                Af = c.y * Af;
            }
        }
    }
    if constexpr (C::BWD && !C::MIXED && !C::QUAD && !C::PROD) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const CT2 c = coef(C::P_NH, u);
            if constexpr (C::ALT) {
                Ab = c.x * Ab;
                Ab1 = c.y * Ab1;
            } else {
                Ab = c.x * Ab;
                Ab = c.y * Ab;
            }
        }
    }
    if constexpr (C::FWD && C::MIXED) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const float4 c = coef4(C::P_F1, u);
            Af32 = (u == 0) ? c.z : c.z * Af32;
            Af32 = c.w * Af32;
        }
    }
    if constexpr (C::BWD && C::MIXED) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const float4 c = coef4(C::P_F2, u);
            Ab32 = c.x * Ab32;
            Ab32 = c.y * Ab32;
        }
    }

    // Complex variants of up to 16 rows per thread under a 256-thread launch
    // bound, and mixed variants of up to 8: each lane's scan multipliers
    // formed once (all systems share them).  The others, with fewer registers
    // to spare, keep the plain scan.
    constexpr bool kPre =
        !C::ALT && ((C::CPLX && R <= 16 && C::kMaxThreads <= 256) || (C::MIXED && !C::CPLX && R <= 8));
    ScanMul<CT> mf{}, mb{};
    ScanMul<float> mf32{}, mb32{};
    if constexpr (kPre && C::FWD && !C::MIXED) mf = scan_multipliers<CT, true>(g, Af);
    if constexpr (kPre && C::BWD && !C::MIXED) mb = scan_multipliers<CT, false>(g, Ab);
    if constexpr (kPre && C::FWD && C::MIXED) mf32 = scan_multipliers<float, true>(g, Af32);
    if constexpr (kPre && C::BWD && C::MIXED) mb32 = scan_multipliers<float, false>(g, Ab32);

    const int sw_me = swz_row<C::SWB>(t), sw_prev = swz_row<C::SWB>(t - 1), sw_next = swz_row<C::SWB>(t + 1);
    const int swo_me = swz_row<C::SWBO>(t);
    const bool has_prev = t > 0, has_next = t < T - 1;
    // rows EPU u .. EPU u + EPU - 1 of plane p of chunk c, in the arithmetic type
    auto unit_rows = [&](const unsigned char* b, int p, int u, int c, int sw, MS (&v)[EPU]) {
        const unsigned char* a = b + in_row(p, u / IB, c) + (((u % IB) ^ sw) << 4);
        if constexpr (ES == 8) {
            const double2 d = *reinterpret_cast<const double2*>(a);
            v[0] = (MS)d.x;
            v[1] = (MS)d.y;
        } else {
            const float4 f = *reinterpret_cast<const float4*>(a);
            v[0] = conv<MS>(f.x);
            v[1] = conv<MS>(f.y);
            v[2] = conv<MS>(f.z);
            v[3] = conv<MS>(f.w);
        }
    };
    // the 16 bytes at `a` from EPU (or, packed complex, 16 / ES) values
    auto put_unit = [&](unsigned char* a, const MS* v) {
        if constexpr (ES == 8) *reinterpret_cast<double2*>(a) = make_double2((double)v[0], (double)v[1]);
        else
            *reinterpret_cast<float4*>(a) =
                make_float4(conv<float>(v[0]), conv<float>(v[1]), conv<float>(v[2]), conv<float>(v[3]));
    };

    const bool win_partial = io.iz0 > 0 || io.iz1 < io.M;

    int bi = 0;        // buffer of this system
    uint32_t par = 0;  // phase parity of its barrier
    for (; sys < nsys; sys += step) {
        unsigned char* cur = buf_at(bi);
        bool ok = mbar_wait_bounded(bar_at(bi), par);
        ok = (W == 1) ? (__all_sync(FULL, ok) != 0) : group_and(g.bar_id, g.nthr, ok);
        if (!ok) {
            if (threadIdx.x == 0) atomicOr(&g_stream_status, kStatusWaitTimeout);
            break;
        }

        // rows s-KL .. s+R+KU-1 of this system
        V be[R + KL + KU];
        // row e of 16-byte unit u of chunk c (both planes when complex)
        auto rows_of = [&](int u, int c, int sw, V (&v)[EPU]) {
            MS re[EPU];
            unit_rows(cur, 0, u, c, sw, re);
            if constexpr (C::CPLX) {
                MS im[EPU];
                unit_rows(cur, 1, u, c, sw, im);
#pragma unroll
                for (int e = 0; e < EPU; ++e) v[e] = V{re[e], im[e]};
            } else {
#pragma unroll
                for (int e = 0; e < EPU; ++e) v[e] = re[e];
            }
        };
#pragma unroll
        for (int u = 0; u < UD; ++u) {
            V v[EPU];
            rows_of(u, t, sw_me, v);
#pragma unroll
            for (int e = 0; e < EPU; ++e) be[KL + EPU * u + e] = v[e];
        }
        if constexpr (KL > 0) {
            V pv[2] = {O::zero(), O::zero()};
            if (has_prev) {  // the last two rows of the chunk before
                V v[EPU];
                rows_of(UD - 1, t - 1, sw_prev, v);
                pv[0] = v[EPU - 2];
                pv[1] = v[EPU - 1];
            }
            be[KL - 1] = pv[1];
            if constexpr (KL > 1) be[0] = pv[0];
        }
        if constexpr (KU > 0) {
            V nv[2] = {O::zero(), O::zero()};
            if (has_next) {  // the first two rows of the chunk after
                V v[EPU];
                rows_of(0, t + 1, sw_next, v);
                nv[0] = v[0];
                nv[1] = v[1];
            }
            be[KL + R] = nv[0];
            if constexpr (KU > 1) be[KL + R + 1] = nv[1];
        }
        if (win_partial) {
#pragma unroll
            for (int i = 0; i < R + KL + KU; ++i) {
                const int64_t row = s - KL + i;
                if (row < io.iz0 || row >= io.iz1) be[i] = O::zero();
            }
        }

        // x = (V A b) scaled by the LU pivots, in place over be[0 .. R)
        if constexpr (C::QUAD) {
#pragma unroll
            for (int q4 = 0; q4 < C::U4; ++q4) {
                float4 wc[NB];
#pragma unroll
                for (int q = 0; q < NB; ++q) wc[q] = coefq(q, q4);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int j = 4 * q4 + e;
                    V acc = O::mul(f4_at(wc[0], e), be[j]);
#pragma unroll
                    for (int q = 1; q < NB; ++q) acc = O::fma(f4_at(wc[q], e), be[j + S * q], acc);
                    be[j] = acc;
                }
            }
        } else {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                CT2 wc[NB];
#pragma unroll
                for (int q = 0; q < NB; ++q) wc[q] = coef(q, u);
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int j = 2 * u + e;
                    V acc = O::mul(e ? wc[0].y : wc[0].x, be[j]);
#pragma unroll
                    for (int q = 1; q < NB; ++q) acc = O::fma(e ? wc[q].y : wc[q].x, be[j + S * q], acc);
                    be[j] = acc;
                }
            }
        }
        V (&x)[R + KL + KU] = be;

        // The load NBUF - 1 systems ahead goes into the buffer of the system
        // before this one, once this warp's stores from it have been read out
        // of shared memory.
        if (sys + (NBUF - 1) * step < nsys && lane == 0) {
            const int pb = (bi == 0) ? NBUF - 1 : bi - 1;
            bulk_wait_read_all();
            issue_load(buf_at(pb), bar_at(pb), sys + (NBUF - 1) * step);
        }

        if constexpr (C::MIXED) {
            // x = M^{-1} g: FP32 solves of the residual, accumulated in FP64
            // (one initial solve, refine_sweeps - 1 refinements).  g = V A b
            // stays in shared memory in place of b (this thread's own rows),
            // so the registers hold only x and the FP32 correction.
            using VF = typename C::VF;
            using OF = VOps<VF>;
            if constexpr (KL + KU > 0) {  // the neighbours' halo reads of b come first
                if (W == 1) __syncwarp();
                else group_bar(g.bar_id, g.nthr);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
#pragma unroll
                for (int p = 0; p < C::NPIN; ++p) {
                    MS v[2];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        if constexpr (C::CPLX) v[e] = p ? x[2 * u + e].y : x[2 * u + e].x;
                        else v[e] = x[2 * u + e];
                    }
                    put_unit(cur + in_row(p, u / IB, t) + (((u % IB) ^ sw_me) << 4), v);
                }
            }
            for (int it = 0; it < op.refine_sweeps; ++it) {
                VF d[R];
                if (it == 0) {
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const float4 f = F1(u);
                        d[2 * u] = OF::mul(f.x, to_f32(x[2 * u]));
                        d[2 * u + 1] = OF::mul(f.y, to_f32(x[2 * u + 1]));
                    }
                } else {
                    // r = g - M x in FP64 (M: unit diagonal, sub al, super cu)
                    V prev, next;
                    group_neighbours<V>(g, x[0], x[R - 1], prev, next);
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const float4 f = F1(u);
                        double2 al = make_double2(0.0, 0.0), cu = make_double2(0.0, 0.0);
                        if constexpr (C::FWD) al = coef(C::P_AL, u);
                        if constexpr (C::BWD) cu = coef(C::P_CU, u);
                        V gu[2];
                        rows_of(u, t, sw_me, gu);
#pragma unroll
                        for (int e = 0; e < 2; ++e) {
                            const int j = 2 * u + e;
                            V mx = x[j];
                            if constexpr (C::FWD) mx = O::fma(e ? al.y : al.x, j > 0 ? x[j - 1] : prev, mx);
                            if constexpr (C::BWD) mx = O::fma(e ? cu.y : cu.x, j < R - 1 ? x[j + 1] : next, mx);
                            d[j] = OF::mul(e ? f.y : f.x, to_f32(O::fma(-1.0, mx, gu[e])));
                        }
                    }
                }
                if constexpr (C::FWD) {
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const float4 f = F1(u);
                        if (u > 0) d[2 * u] = OF::fma(f.z, d[2 * u - 1], d[2 * u]);
                        d[2 * u + 1] = OF::fma(f.w, d[2 * u], d[2 * u + 1]);
                    }
                    VF pin;
                    if constexpr (kPre) pin = group_affine_scan_pre<VF, float, true>(g, mf32, d[R - 1]);
                    else pin = group_affine_scan<VF, float, true>(g, Af32, d[R - 1]);
                    float p = 1.0f;
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const float4 f = F1(u);
                        p = f.z * p;
                        d[2 * u] = OF::fma(p, pin, d[2 * u]);
                        p = f.w * p;
                        d[2 * u + 1] = OF::fma(p, pin, d[2 * u + 1]);
                    }
                }
                if constexpr (C::BWD) {
#pragma unroll
                    for (int u = U - 1; u >= 0; --u) {
                        const float2 f = F2(u);
                        if (u < U - 1) d[2 * u + 1] = OF::fma(f.y, d[2 * u + 2], d[2 * u + 1]);
                        d[2 * u] = OF::fma(f.x, d[2 * u + 1], d[2 * u]);
                    }
                    VF q;
                    if constexpr (kPre) q = group_affine_scan_pre<VF, float, false>(g, mb32, d[0]);
                    else q = group_affine_scan<VF, float, false>(g, Ab32, d[0]);
                    float p = 1.0f;
#pragma unroll
                    for (int u = U - 1; u >= 0; --u) {
                        const float2 f = F2(u);
                        p = f.y * p;
                        d[2 * u + 1] = OF::fma(p, q, d[2 * u + 1]);
                        p = f.x * p;
                        d[2 * u] = OF::fma(p, q, d[2 * u]);
                    }
                }
                if (it == 0) {
#pragma unroll
                    for (int j = 0; j < R; ++j) x[j] = to_f64(d[j]);
                } else {
#pragma unroll
                    for (int j = 0; j < R; ++j) x[j] = O::add(x[j], to_f64(d[j]));
                }
            }
        }
        if constexpr (C::FWD && !C::MIXED && C::ALT) {
            // the same per system: z_j = x_j - l_j z_{j-2}; both systems' chunk
            // couplings in one paired scan
#pragma unroll
            for (int u = 1; u < U; ++u) {
                const CT2 c = coef(C::P_NL, u);
                x[2 * u] = O::fma(c.x, x[2 * u - 2], x[2 * u]);
                x[2 * u + 1] = O::fma(c.y, x[2 * u - 1], x[2 * u + 1]);
            }
            const double2 pin = group_affine_scan2<true>(g, make_double2(Af, Af1), make_double2(x[R - 2], x[R - 1]));
            const V pin0 = pin.x, pin1 = pin.y;
            CT p0 = 1, p1 = 1;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const CT2 c = coef(C::P_NL, u);
                p0 = c.x * p0;
                x[2 * u] = O::fma(p0, pin0, x[2 * u]);
                p1 = c.y * p1;
                x[2 * u + 1] = O::fma(p1, pin1, x[2 * u + 1]);
            }
        }
        if constexpr (C::FWD && C::QUAD) {
            // z_j = x_j - l_j z_{j-1} within the chunk, then the coupling from
            // the preceding chunks times the stored product of -l up to row j
#pragma unroll
            for (int q4 = 0; q4 < C::U4; ++q4) {
                const float4 c = coefq(C::P_NL, q4);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int j = 4 * q4 + e;
                    if (j > 0) x[j] = O::fma(f4_at(c, e), x[j - 1], x[j]);
                }
            }
            V pin;
            if constexpr (kPre) pin = group_affine_scan_pre<V, CT, true>(g, mf, x[R - 1]);
            else pin = group_affine_scan<V, CT, true>(g, Af, x[R - 1]);
#pragma unroll
            for (int q4 = 0; q4 < C::U4; ++q4) {
                const float4 pl = coefq(C::P_PL, q4);
#pragma unroll
                for (int e = 0; e < 4; ++e) x[4 * q4 + e] = O::fma(f4_at(pl, e), pin, x[4 * q4 + e]);
            }
        }
        if constexpr (C::FWD && !C::MIXED && !C::ALT && !C::QUAD) {
            // z_j = x_j - l_j z_{j-1} within the chunk, then add the coupling
            // from the preceding chunks scaled by prod_{k<=j}(-l_k)
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const CT2 c = coef(C::P_NL, u);
                if (u > 0) x[2 * u] = O::fma(c.x, x[2 * u - 1], x[2 * u]);
                x[2 * u + 1] = O::fma(c.y, x[2 * u], x[2 * u + 1]);
            }
            V pin;
            if constexpr (kPre) pin = group_affine_scan_pre<V, CT, true>(g, mf, x[R - 1]);
            else pin = group_affine_scan<V, CT, true>(g, Af, x[R - 1]);
            if constexpr (C::PROD) {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const CT2 pl = coef(C::P_PL, u);
                    x[2 * u] = O::fma(pl.x, pin, x[2 * u]);
                    x[2 * u + 1] = O::fma(pl.y, pin, x[2 * u + 1]);
                }
            } else {
                CT p = 1;
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const CT2 c = coef(C::P_NL, u);
                    p = c.x * p;
                    x[2 * u] = O::fma(p, pin, x[2 * u]);
                    p = c.y * p;
                    x[2 * u + 1] = O::fma(p, pin, x[2 * u + 1]);
                }
            }
        }
        if constexpr (C::BWD && !C::MIXED && C::ALT) {
#pragma unroll
            for (int u = U - 2; u >= 0; --u) {
                const CT2 c = coef(C::P_NH, u);
                x[2 * u + 1] = O::fma(c.y, x[2 * u + 3], x[2 * u + 1]);
                x[2 * u] = O::fma(c.x, x[2 * u + 2], x[2 * u]);
            }
            const double2 q = group_affine_scan2<false>(g, make_double2(Ab, Ab1), make_double2(x[0], x[1]));
            const V q0 = q.x, q1 = q.y;
            CT p0 = 1, p1 = 1;
#pragma unroll
            for (int u = U - 1; u >= 0; --u) {
                const CT2 c = coef(C::P_NH, u);
                p1 = c.y * p1;
                x[2 * u + 1] = O::fma(p1, q1, x[2 * u + 1]);
                p0 = c.x * p0;
                x[2 * u] = O::fma(p0, q0, x[2 * u]);
            }
        }
        if constexpr (C::BWD && C::QUAD) {
#pragma unroll
            for (int q4 = C::U4 - 1; q4 >= 0; --q4) {
                const float4 c = coefq(C::P_NH, q4);
#pragma unroll
                for (int e = 3; e >= 0; --e) {
                    const int j = 4 * q4 + e;
                    if (j < R - 1) x[j] = O::fma(f4_at(c, e), x[j + 1], x[j]);
                }
            }
            V q;
            if constexpr (kPre) q = group_affine_scan_pre<V, CT, false>(g, mb, x[0]);
            else q = group_affine_scan<V, CT, false>(g, Ab, x[0]);
#pragma unroll
            for (int q4 = 0; q4 < C::U4; ++q4) {
                const float4 ph = coefq(C::P_PH, q4);
#pragma unroll
                for (int e = 0; e < 4; ++e) x[4 * q4 + e] = O::fma(f4_at(ph, e), q, x[4 * q4 + e]);
            }
        }
        if constexpr (C::BWD && !C::MIXED && !C::ALT && !C::QUAD) {
#pragma unroll
            for (int u = U - 1; u >= 0; --u) {
                const CT2 c = coef(C::P_NH, u);
                if (u < U - 1) x[2 * u + 1] = O::fma(c.y, x[2 * u + 2], x[2 * u + 1]);
                x[2 * u] = O::fma(c.x, x[2 * u + 1], x[2 * u]);
            }
            V q;
            if constexpr (kPre) q = group_affine_scan_pre<V, CT, false>(g, mb, x[0]);
            else q = group_affine_scan<V, CT, false>(g, Ab, x[0]);
            if constexpr (C::PROD) {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const CT2 ph = coef(C::P_PH, u);
                    x[2 * u] = O::fma(ph.x, q, x[2 * u]);
                    x[2 * u + 1] = O::fma(ph.y, q, x[2 * u + 1]);
                }
            } else {
                CT p = 1;
#pragma unroll
                for (int u = U - 1; u >= 0; --u) {
                    const CT2 c = coef(C::P_NH, u);
                    p = c.y * p;
                    x[2 * u + 1] = O::fma(p, q, x[2 * u + 1]);
                    p = c.x * p;
                    x[2 * u] = O::fma(p, q, x[2 * u]);
                }
            }
        }
        if (C::SV != SV_NONE && s == 0) x[0] = O::mul(op.scaleC, x[0]);
        if constexpr (C::SCALE && C::QUAD) {
#pragma unroll
            for (int q4 = 0; q4 < C::U4; ++q4) {
                const float4 c = coefq(C::P_SC, q4);
#pragma unroll
                for (int e = 0; e < 4; ++e) x[4 * q4 + e] = O::mul(f4_at(c, e), x[4 * q4 + e]);
            }
        }
        if constexpr (C::SCALE && !C::QUAD) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const CT2 c = coef(C::P_SC, u);
                x[2 * u] = O::mul(c.x, x[2 * u]);
                x[2 * u + 1] = O::mul(c.y, x[2 * u + 1]);
            }
        }

        // Stage the result in place.  Every thread of the group has read its
        // input: the solve's scans are group barriers; without a solve, wait.
        if constexpr (C::SV == SV_NONE) {
            if (W > 1) group_bar(g.bar_id, g.nthr);
        }
        __syncwarp();
        // output unit uo holds EPUO rows (packed complex: re, im of each)
        auto out_unit = [&](int p, int uo) -> unsigned char* {
            return cur + out_row(p, uo / IBO, t) + (((uo % IBO) ^ swo_me) << 4);
        };
        if constexpr (C::OPK) {
#pragma unroll
            for (int uo = 0; uo < UO; ++uo) {
                MS v[4];
#pragma unroll
                for (int e = 0; e < C::EPUO; ++e) {
                    v[2 * e] = x[C::EPUO * uo + e].x;
                    v[2 * e + 1] = x[C::EPUO * uo + e].y;
                }
                put_unit(out_unit(0, uo), v);
            }
        } else {
#pragma unroll
            for (int uo = 0; uo < UO; ++uo) {
#pragma unroll
                for (int p = 0; p < C::NPOUT; ++p) {
                    MS v[4];
#pragma unroll
                    for (int e = 0; e < EPU; ++e) {
                        if constexpr (C::CPLX) v[e] = p ? x[EPU * uo + e].y : x[EPU * uo + e].x;
                        else v[e] = x[EPU * uo + e];
                    }
                    put_unit(out_unit(p, uo), v);
                }
            }
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) issue_store(cur, sys);
        if (++bi == NBUF) {
            bi = 0;
            par ^= 1u;
        }
    }
    if (lane == 0) bulk_wait_all();
}

}  // namespace pfb
