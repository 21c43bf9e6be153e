// api.cpp -- the C ABI of include/pfsolve_b200.h: plan creation, launch, apps
// library and fused chains.  Host logic mirrors PfSolve's plan/application
// layer for the JW path (PfSolve/pfSolve_AppManagement/*,
// PfSolve/pfSolve_PlanManagement/pfSolve_Plans/pfSolve_Plan_JonesWorland.h)
// without runtime code generation: every kernel variant is precompiled.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <tuple>
#include <vector>

#include "../../include/pfsolve_b200.h"
#include "jw_variants.h"
#include "plan.h"

using namespace pfb;

namespace {

std::atomic<uint64_t> g_launches{0};
std::atomic<uint64_t> g_stream_launches{0};

enum AppKind { APP_JW = 1, APP_DGBMV = 2, APP_BLOCK = 3, APP_DCT = 4 };

constexpr int64_t kMaxRows = 4096;       // one CTA group per system (<= 8 warps x 32 x 16 rows)
constexpr int64_t kMaxRowsLong = 65536;  // JW apps: up to 64 slices of 1024 rows per system (single pass)

struct AppState {
    AppKind kind;
    int num_sms = 0;
    int device = 0;
    // JW / dgbmv plan
    int R = 0, W = 1, G = 1;
    int mvj = MVJ_NONE, sv = SV_NONE, KL = 0, KU = 0;
    int prec = 0;           // PREC_*: FP64, FP32 solve + FP64 refinement, dd, FP32, FP64 on FP32 storage
    bool R_fixed = false;   // rows per thread requested by the caller
    int refine_sweeps = 1;  // FP32 solves per system in the mixed mode
    const JwVariant* variant = nullptr;
    int max_blocks = 0;  // resident CTAs over the whole GPU
    // streaming variant (FP64, TMA-staged systems), used when a launch's
    // buffers allow it; `variant` serves the other launches
    const StreamVariant* stream_v = nullptr;
    int stream_G = 0, stream_max_blocks = 0;
    int stream_nbuf = 2;  // staging buffers per group
    int nbuf_req = 0;     // caller's staging buffers per group (0: choose)
    // long systems (N > 4096): two passes over slices (default), or one
    // cluster of CTAs per system (kernelPath 2)
    const LongVariant* long_v = nullptr;
    int long_NS = 0, long_grid = 0;
    double* long_red = nullptr;  // per (system, slice) records, then per-slice constants
    unsigned* long_flags = nullptr;  // single pass: per (system, slice) publication flags
    unsigned long_epoch = 0;         // single pass: flag value of the latest launch
    double2* dct_tables = nullptr;   // DCT step: twiddles, then pre/post factors (2N values)
    int dct_logn = 0;
    bool long_single = false;        // the plan's form: single pass, else pass 1, carries, pass 2
    int long_mode = 0;               // kernelPath: 0 two passes where M allows (else single), 3 two, 4 single
    const LongVariant* long_v_fb = nullptr;  // single-pass fallback for rows no tensor map describes
    int long_grid_fb = 0;
    int64_t long_batch = 0;      // systems the records hold
    int64_t plan_batch = 0;      // right-hand sides of the plan (size[1] * size[2])
    bool cluster_only = false;   // kernelPath 2
    const ClusterVariant* cluster_v = nullptr;
    int cluster_max = 0;
    int R_req = 0;           // caller's rows per thread (0: choose)
    bool no_stream = false;  // kernelPath 1
    bool no_tbl = false;     // register-coefficient variants only
    uint64_t dg_skip = 0;    // dgbmv with ALT_dgbmv: bands dropped (bit j: band j)
    // ALT stride-2 mode: even and odd rows solved as two systems on the group
    // kernel (lanes x rows of the reference's ALT band layout)
    bool alt = false;
    int64_t alt_T = 0, alt_R = 0;
    // K consecutive steps (numConsecutiveJWIterations > 1): one kernel
    int K = 1;
    const StepsVariant* steps_v = nullptr;
    int steps_W = 1, steps_G = 1, steps_max_blocks = 0, steps_nbuf = 1;
    int64_t steps_r = 1;  // rows per lane of the reference's band order
    // bidiagonal kinds: one system per lane, all steps in one sweep (used when
    // a launch's buffers allow the TMA boxes), NW warps per CTA at most
    const SeqStepsVariant* seq_v = nullptr;
    int seq_NW = 0;
    // fused-chain plans made with this JW app, by operator shape
    struct ChainPlan {
        int KL, KU, sv, LIN, LOUT, SCALE;
        const JwVariant* variant;
        int R, W, G, max_blocks;
        const StreamVariant* stream_v;
        int stream_G, stream_max_blocks, stream_nbuf;
    };
    std::vector<ChainPlan> chain_plans;
    // streams
    uint64_t stream_counter = 0;
    cudaEvent_t* events = nullptr;
};

AppState* st(PfSolveApplication* app) { return static_cast<AppState*>(app->internal); }

// The kernel instance of the calling thread's most recent launch
// (PfSolveGetLastLaunch).
thread_local PfSolveLaunchInfo g_last_launch;

void record_launch(int kernel, int R, int W, int G, int KL, int KU, int sv, int lin, int lout, int scale, int prec,
                   int alt, int64_t grid)
{
    PfSolveLaunchInfo& i = g_last_launch;
    i.kernel = kernel;
    i.rowsPerThread = R;
    i.warpsPerSystem = W;
    i.groupsPerCTA = G;
    i.bandsBelow = KL;
    i.bandsAbove = KU;
    i.solve = sv;
    i.layoutIn = lin;
    i.layoutOut = lout;
    i.scale = scale;
    i.precision = prec;
    i.alt = alt;
    i.gridCTAs = grid;
}

}  // namespace

void pfb::note_launch(bool streaming)
{
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (streaming) g_stream_launches.fetch_add(1, std::memory_order_relaxed);
}

namespace {

// Keep-window of PfConfigureZeropad (pfSolve_KernelsLevel0/pfSolve_Zeropad.h:306-377)
// as a half-open row range.  Launch-time windows keep [z0, z1); plan-time
// windows treat 0 as "unbounded".
void keep_window(bool runtime, int64_t z0, int64_t z1, int64_t& lo, int64_t& hi)
{
    const int64_t BIG = INT64_MAX / 4;
    if (runtime) { lo = z0; hi = z1; return; }
    lo = z0 ? z0 : 0;
    hi = z1 ? z1 : BIG;
}

// Default rows per thread: 4 keeps the data of a coefficient-table variant
// within 128 registers (two 256-thread groups per SM); longer systems need
// more rows per thread to stay within 8 warps per system.
int pick_rows_per_thread(int64_t M, int requested)
{
    if (requested == 2 || requested == 4 || requested == 8 || requested == 16) return requested;
    if (M <= 64) return 2;
    if (M <= 1024) return 4;
    if (M <= 2048) return 8;
    return 16;
}

// Streaming variant for M rows: rows per thread R (the caller's choice, else
// the compiled R whose groups leave the fewest idle rows, 16 first), W warps
// per system, and the most groups per CTA that fit shared memory.  ALT: M
// counts the rows of a row set (both systems).
bool choose_stream(AppState* s, int64_t M, int LIN, int LOUT, int SCALE, bool alt = false)
{
    s->stream_v = nullptr;
    if ((s->prec != PREC_F64 && s->prec != PREC_MIXED && !prec_f32_storage(s->prec)) || s->no_stream) return false;
    int cand[3][2];
    int n = 0;
    const int prefs[3] = {16, 32, 8};
    for (int R : prefs) {
        if (s->R_req && R != s->R_req) continue;
        const int64_t W = (M + 32 * (int64_t)R - 1) / (32 * (int64_t)R);
        if (M % R != 0 || !(W == 1 || W == 2 || W == 4)) continue;
        cand[n][0] = R;
        cand[n][1] = (int)W;
        n++;
    }
    // fewest idle rows first (stable: keeps the preference order on ties)
    for (int i = 1; i < n; ++i)
        for (int j = i; j > 0; --j) {
            const int64_t a = 32LL * cand[j][1] * cand[j][0] - M, b = 32LL * cand[j - 1][1] * cand[j - 1][0] - M;
            if (a >= b) break;
            std::swap(cand[j], cand[j - 1]);
        }
    for (int i = 0; i < n; ++i) {
        const StreamVariant* v =
            find_stream_variant(cand[i][0], cand[i][1], s->KL, s->KU, s->sv, LIN, LOUT, SCALE, s->prec, alt);
        if (!v) continue;
        const int T = 32 * v->W;
        // Most groups first, two staging buffers per group -- three for FP32
        // storage and arithmetic where they fit beside as many groups -- (a
        // caller's request: the most groups that fit with it).  Measured at
        // N = 512 (131 072 systems): 3 or 4 buffers per group were no faster
        // for FP64, the mixed mode or FP64 arithmetic on FP32 storage, 3 %
        // faster for FP32 (its 2-KB systems, solved fastest, need more of them
        // in flight), and where they cost groups (the config-2 chain) much
        // slower.
        auto fits = [&](int G, int nb, int* blocks) {
            const size_t smem = v->smem_bytes(G, nb);
            if (smem > 227 * 1024 || !allow_max_smem(v->func)) return false;
            return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, v->func, T * G, smem) == cudaSuccess &&
                   *blocks >= 1;
        };
        const bool req = s->nbuf_req >= 2 && s->nbuf_req <= kStMaxBuffers;
        for (int G = std::min(v->max_threads / T, 15); G >= 1; --G) {
            int blocks = 0;
            int nb = req ? s->nbuf_req : 2;
            if (!req && s->prec == PREC_F32 && fits(G, 3, &blocks)) nb = 3;
            if (!fits(G, nb, &blocks)) continue;
            s->stream_v = v;
            s->stream_G = G;
            s->stream_nbuf = nb;
            s->stream_max_blocks = blocks * s->num_sms;
            return true;
        }
    }
    cudaGetLastError();
    return false;
}

// Long-system variant for real systems: the first compiled shape that fits
// the given form.  Both forms take any M: a last partial chunk of R rows moves
// outside the TMA boxes, by its thread's plain loads and stores (measured at
// M = 4 104: 16 rows per thread with a partial chunk, 0.816 ms, against 8 rows
// per thread and whole chunks, 0.884 ms).
const LongVariant* pick_long(AppState* s, int64_t M, bool single, int* NS_out, int* grid_out,
                             const LongVariant* like = nullptr)
{
    for (int shape = 0; shape < kLongShapes; ++shape) {
        const LongVariant* v = find_long_variant(shape, s->KL, s->KU, s->sv);
        if (!v) return nullptr;
        // a fallback shares the plan's records and tables: same slices
        if (like && (v->R != like->R || v->W != like->W || v->S != like->S || v->tbl_bytes != like->tbl_bytes))
            continue;
        const int b = v->blocks_per_sm(single);
        if (b < 1) continue;
        const int NS = (int)((M + v->S - 1) / v->S);
        if (single && NS > kLongMaxSlices) continue;
        const int64_t res = (int64_t)b * s->num_sms;
        *NS_out = NS;
        if (single) {
            // CTAs in whole multiples of NS, at most one CTA's worth of systems each
            const int64_t per_slice =
                std::max<int64_t>(1, std::min<int64_t>(res / NS, (s->plan_batch + v->G - 1) / v->G));
            *grid_out = (int)(per_slice * NS);
        } else {
            // the solve passes split the (slice, system) items evenly over
            // every resident CTA, at least a group's worth each
            const int64_t items = (int64_t)NS * s->plan_batch;
            *grid_out = (int)std::max<int64_t>(1, std::min<int64_t>(res, (items + v->G - 1) / v->G));
        }
        return v;
    }
    return nullptr;
}

// Long systems (M > 4096, real FP64).  kernelPath 0: two passes (measured
// faster than the single pass at every length), with a single-pass fallback
// for launches whose rows no tensor map can describe.  kernelPath 3: two
// passes only; 4: the single pass only.  The per-(system, slice) records are allocated for the plan's
// right-hand sides.
bool choose_long(AppState* s, int64_t M, int LIN, int LOUT, int SCALE)
{
    s->long_v = nullptr;
    s->long_v_fb = nullptr;
    if (s->prec != PREC_F64 || s->no_stream || s->cluster_only || LIN != LAY_REAL || LOUT != LAY_REAL || SCALE ||
        s->plan_batch < 1)
        return false;
    int NS = 0, grid = 0, NSf = 0, gridf = 0;
    const LongVariant* v = nullptr;
    const LongVariant* fb = nullptr;
    if (s->long_mode != 4) v = pick_long(s, M, false, &NS, &grid);
    if (v && s->long_mode == 0) {
        fb = pick_long(s, M, true, &NSf, &gridf, v);
        if (!fb || NSf != NS) v = fb = nullptr;  // no fallback of the same slices: the single pass alone
    }
    bool single = false;
    if (!v && s->long_mode != 3) {
        v = pick_long(s, M, true, &NS, &grid);
        single = true;
    }
    if (!v) return false;
    // records, slice constants, slice tables, PASS 1 weights (16 bytes per
    // row), then the single pass's flags (4 bytes per system and slice)
    const size_t fbytes = (size_t)s->plan_batch * NS * sizeof(unsigned);
    const size_t bytes = ((size_t)s->plan_batch * NS * 8 + (size_t)NS * 8) * sizeof(double) +
                         (size_t)NS * v->tbl_bytes + (size_t)NS * v->S * 16 + fbytes;
    if (cudaMalloc(&s->long_red, bytes) != cudaSuccess) {
        cudaGetLastError();
        s->long_red = nullptr;
        return false;
    }
    s->long_flags = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(s->long_red) + bytes - fbytes);
    if (cudaMemset(s->long_flags, 0, fbytes) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(s->long_red);
        s->long_red = nullptr;
        return false;
    }
    s->long_v = v;
    s->long_single = single;
    s->long_NS = NS;
    s->long_grid = grid;
    s->long_v_fb = fb;
    s->long_grid_fb = gridf;
    s->long_batch = s->plan_batch;
    return true;
}

// Cluster variant for long real systems: C CTAs of 2048 rows, C the smallest
// compiled count that covers M (rows per thread 8: M must be a multiple of 8).
bool choose_cluster(AppState* s, int64_t M, int LIN, int LOUT, int SCALE)
{
    s->cluster_v = nullptr;
    if (s->prec != PREC_F64 || s->no_stream || LIN != LAY_REAL || LOUT != LAY_REAL || SCALE || M % 8 != 0)
        return false;
    for (int C : {3, 4, 6, 8}) {
        if ((int64_t)C * 2048 < M) continue;
        const ClusterVariant* v = find_cluster_variant(C, s->KL, s->KU, s->sv);
        if (!v) return false;
        if (!allow_max_smem(v->func)) return false;
        const int n = v->max_clusters(v->smem_bytes);
        if (n < 1) return false;
        s->cluster_v = v;
        s->cluster_max = n;
        return true;
    }
    return false;
}

// Rows per lane of the reference's band order for a K-step plan: from M + K - 1
// rows when the steps grow the system (upperBanded 0), else from M
// (pfSolve_Plan_JonesWorland.h:276-283, 311-314, 342-346).
int64_t steps_band_registers(int64_t M, int ub, int K)
{
    const int64_t tm = ub ? M : M + K - 1;
    int64_t warp = 64 * ((tm + 1023) / 1024);
    if (tm < 512) warp = 32;
    if (warp < 32) warp = 32;
    if (warp % 32) warp = 32 * ((warp + 31) / 32);
    const int64_t r = (tm + warp - 1) / warp;
    return r < 1 ? 1 : r;
}

// K-step plan (pfSolve_KernelsLevel2/pfSolve_JonesWorland.h:108-374).  Defined
// combinations: upperBanded 0/1 with jw_type % 10 in {0, 1, 2}; upperBanded 2
// with jw_type % 10 == 3 and K == 2 (for K > 2 the reference multiplies the
// middle steps by a diagonal it never reloads, pfSolve_ReadWrite.h:1650; the
// same holds for jw_type % 10 == 3 with upperBanded 0/1).
// Rows per TMA box of the K-step sweep kernel: 16 (128 bytes of each system
// per box) up to 6 steps, 8 above, where the step tables leave room for too
// few warps of 16-row buffers (measured at N = 512, 131 072 RHS with 16-row
// boxes against 8: K = 2, 4 4-7 % faster; K = 5, 6 (three buffers a warp)
// 4 % faster; K = 8 9 % slower).
static int seq_chunk_rows(int K) { return K <= 6 ? 16 : 8; }

PfSolveResult plan_steps(AppState* s, const PfSolveConfiguration& c)
{
    const int K = c.numConsecutiveJWIterations, ub = c.upperBanded, jwt = c.jw_type % 10;
    if (K > kMaxSteps) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    if (s->prec != PREC_F64 || c.mixedPrecisionRefinement) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    if (ub == 2 ? (jwt != 3 || K != 2) : !(jwt == 0 || jwt == 1 || jwt == 2)) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    if (c.useMultipleInputBuffers > 1 && c.useMultipleInputBuffers < K) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    // launch-time band offsets: the reference's plan creation fails (the
    // process crashes) for K > 1, so there is no behaviour to follow
    if (c.jw_control_bitmask & (RUNTIME_OFFSETM | RUNTIME_OFFSETV)) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    const int64_t M = c.M_size, Mmax = ub ? M : M + K - 1, Mout = ub ? M - K + 1 : M + K - 1;
    if (Mout < 1) return PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH;
    if (Mmax > kMaxRows) return PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH;
    s->K = K;
    s->steps_nbuf = c.useMultipleInputBuffers > 1 ? c.useMultipleInputBuffers : 1;
    s->steps_r = steps_band_registers(M, ub, K);
    const int MV = jwt != 2;
    const int KL = (MV && ub == 0) ? 1 : 0, KU = (MV && ub == 1) ? 1 : 0;
    const int SV = ub == 2 ? SV_TRI : (jwt == 1 ? SV_NONE : (ub == 1 ? SV_LOWER : SV_UPPER));
    int Rs[3] = {4, 8, 16};
    int n = 3;
    if (c.rowsPerThread == 4 || c.rowsPerThread == 8 || c.rowsPerThread == 16) {
        Rs[0] = c.rowsPerThread;
        n = 1;
    }
    int maxopt = 0;
    cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device);
    if (ub != 2 && c.kernelPath != 1) {
        const int64_t Mtab = ub ? M : Mout;
        for (int CH : {seq_chunk_rows(K), 8}) {
            const SeqStepsVariant* v = find_seq_steps_variant(ub, MV, SV != SV_NONE, K, CH);
            const int64_t fixed = (int64_t)seq_steps_smem_bytes(K, Mtab, 0, CH);
            const int64_t per_warp = (int64_t)seq_steps_smem_bytes(K, Mtab, 1, CH) - fixed;
            int nw = (int)std::min<int64_t>(v ? v->max_threads / 32 : 0, ((int64_t)maxopt - fixed) / per_warp);
            if (v && nw >= 4 && allow_max_smem(v->func)) {
                int blocks = 0;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, v->func, 32 * nw,
                                                                  seq_steps_smem_bytes(K, Mtab, nw, CH)) ==
                        cudaSuccess &&
                    blocks >= 1) {
                    s->seq_v = v;
                    s->seq_NW = nw;
                    break;
                }
            }
            cudaGetLastError();
        }
    }
    for (int i = 0; i < n; ++i) {
        const int R = Rs[i];
        const int64_t W = (Mmax + 32 * (int64_t)R - 1) / (32 * (int64_t)R);
        // at most 8 warps per system; 4 rows per thread only for one warp
        if (W > 8 || (n == 3 && R == 4 && W > 1) || (n == 3 && R == 8 && W > 8)) continue;
        const StepsVariant* v = find_steps_variant(R, KL, KU, SV, MV);
        if (!v) continue;
        const int maxthr = R >= 16 ? 256 : 512;
        if (32 * W > maxthr) continue;
        for (int G = std::min(maxthr / (32 * (int)W), 15); G >= 1; --G) {  // named barriers 1..15
            const size_t smem = v->smem_bytes(K, (int)W, G);
            if ((int)smem > maxopt) continue;
            if (smem > 48 * 1024 && !allow_max_smem(v->func)) continue;
            int blocks = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, v->func, 32 * (int)W * G, smem) != cudaSuccess ||
                blocks < 1)
                continue;
            s->steps_v = v;
            s->steps_W = (int)W;
            s->steps_G = G;
            s->steps_max_blocks = blocks * s->num_sms;
            return PFSOLVE_SUCCESS;
        }
    }
    cudaGetLastError();
    // the step tables do not fit shared memory: a sweep-only plan, else none
    return s->seq_v ? PFSOLVE_SUCCESS : PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
}

PfSolveResult finish_variant(AppState* s, int64_t M, int LIN, int LOUT, int SCALE);

// ALT stride-2 mode (jw_type / 100 % 10 == 1, pfSolve_Plan_JonesWorland.h:265):
// the even and the odd rows of a system are two independent systems with
// neighbours r -+ 2 (the reference's lanes split in two halves,
// pfSolve_TridiagonalSolve.h:1319-1330, 1622-1644), bands in its ALT register
// layout R T entries apart (pfSolve_JonesWorland.h:209-222, 262-271,
// pfSolve_ReadWrite.h:1705-1711).  K = 1; plan-time band offsets only (the
// reference rescales only those); FP64 or FP32 solve + FP64 refinement.
PfSolveResult plan_alt(AppState* s, const PfSolveConfiguration& c, int base_prec)
{
    if (c.numConsecutiveJWIterations > 1 || base_prec != PREC_F64) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    if (c.jw_control_bitmask & (RUNTIME_OFFSETM | RUNTIME_OFFSETV)) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    if (c.upperBanded < 0 || c.upperBanded > 2) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    const int64_t M = c.M_size;
    if (M < 2 || (M + 1) / 2 > kMaxRows) return PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH;
    JwLayout L;
    if (!jw_layout(c, false, false, 0, 0, L)) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    int64_t warp = 64 * ((M + 1023) / 1024);
    if (M < 512) warp = 32;
    if (warp % 32) warp = 32 * ((warp + 31) / 32);
    s->alt = true;
    s->alt_T = warp;
    s->alt_R = (M + warp - 1) / warp;
    s->mvj = L.mvj;
    s->sv = L.sv;
    s->prec = (c.mixedPrecisionRefinement > 0 && L.sv != SV_NONE) ? 1 : 0;
    s->refine_sweeps = 1 + c.mixedPrecisionRefinement;
    s->KL = (L.mvj == MVJ_LOWER) ? 1 : 0;
    s->KU = (L.mvj == MVJ_UPPER) ? 1 : 0;
    const int64_t n0 = (M + 1) / 2;  // rows of the even system
    s->R = pick_rows_per_thread(n0, c.rowsPerThread);
    s->R_fixed = c.rowsPerThread != 0 && c.rowsPerThread != 32;
    s->R_req = c.rowsPerThread;
    s->no_stream = true;  // group kernel: per-group parity, stride-2 rows
    s->no_tbl = true;     // the two parities have different coefficients
    const PfSolveResult r = finish_variant(s, n0, LAY_REAL, LAY_REAL, 0);
    if (r != PFSOLVE_SUCCESS || !s->variant) return r == PFSOLVE_SUCCESS ? PFSOLVE_ERROR_UNSUPPORTED_COMBINATION : r;
    // FP64: the streaming kernel stages whole row sets and solves their two
    // systems together; the group kernel above takes the launches it cannot
    // (partial output windows, unaligned rows) and kernelPath 1.
    s->no_stream = c.kernelPath == 1;
    if (s->prec == PREC_F64) choose_stream(s, M, LAY_REAL, LAY_REAL, 0, true);
    return PFSOLVE_SUCCESS;
}

// Pick the kernel variant and launch shape for M rows: register variants
// first, then coefficient-table variants (FP64); rows per thread from the
// caller's choice (s->R) first, then the other compiled choices.
PfSolveResult finish_variant(AppState* s, int64_t M, int LIN, int LOUT, int SCALE)
{
    // Double-double: the table form first (16 rows per thread where a system
    // fits one warp, else 8), then the register form (the caller's rows per
    // thread: those, in either form).
    if ((s->prec == PREC_DD || s->prec == PREC_DD_F64MEM) && !s->no_tbl && LIN == LAY_REAL && LOUT == LAY_REAL &&
        !SCALE) {
        const int cand[3][2] = {{16, 1}, {8, 1}, {4, 1}};
        for (const auto& rc : cand) {
            const int R = rc[0];
            if (s->R_req && R != s->R_req) continue;
            const int64_t W = (M + 32 * (int64_t)R - 1) / (32 * (int64_t)R);
            if (W < 1 || W > 4 || (R == 16 && W > 1 && !s->R_req)) continue;
            const JwVariant* v = find_jw_variant(R, s->KL, s->KU, s->sv, LIN, LOUT, SCALE, s->prec, 1);
            if (!v || 32 * W > v->max_threads) continue;
            int G = 0, maxb = 0;
            if (!choose_groups(v, (int)W, s->num_sms, G, maxb)) continue;
            s->variant = v;
            s->R = R;
            s->W = (int)W;
            s->G = G;
            s->max_blocks = maxb;
            return PFSOLVE_SUCCESS;
        }
    }
    const int order[4] = {s->R, 8, 4, 16};
    // The caller's rows per thread first; when the group kernel has no such
    // variant (the choice is then the streaming kernel's), any other.
    for (int pass = 0; pass < 2; ++pass)
    for (int tbl = 0; tbl <= (s->prec == 0 && !s->no_tbl ? 1 : 0); ++tbl) {
        for (int oi = 0; oi < 4; ++oi) {
            const int R = order[oi];
            if (oi > 0 && (R == s->R || (s->R_fixed && pass == 0))) continue;
            const JwVariant* v = find_jw_variant(R, s->KL, s->KU, s->sv, LIN, LOUT, SCALE, s->prec, tbl);
            if (!v) continue;
            const int64_t W = (M + 32 * (int64_t)R - 1) / (32 * (int64_t)R);
            if (W < 1 || W > 8 || 32 * W > v->max_threads) continue;
            int G = 0, maxb = 0;
            if (!choose_groups(v, (int)W, s->num_sms, G, maxb)) continue;
            s->variant = v;
            choose_stream(s, M, LIN, LOUT, SCALE);
            s->R = R;
            s->W = (int)W;
            s->G = G;
            s->max_blocks = maxb;
            return PFSOLVE_SUCCESS;
        }
    }
    // No group-kernel variant fits: a streaming-only plan (or, for long
    // systems, a cluster plan), whose launches need buffers those kernels can
    // take.
    s->variant = nullptr;
    if (choose_stream(s, M, LIN, LOUT, SCALE)) return PFSOLVE_SUCCESS;
    if (M > kMaxRows && choose_long(s, M, LIN, LOUT, SCALE)) return PFSOLVE_SUCCESS;
    if (M > kMaxRows && choose_cluster(s, M, LIN, LOUT, SCALE)) return PFSOLVE_SUCCESS;
    // nothing compiled fits: distinguish "too long" from "not compiled"
    for (int R : {2, 4, 8, 16})
        if ((M + 32 * (int64_t)R - 1) / (32 * (int64_t)R) <= 8) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    return PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH;
}

cudaStream_t pick_stream(PfSolveApplication* app)
{
    PfSolveConfiguration& c = app->configuration;
    AppState* s = st(app);
    if (!c.stream || c.num_streams == 0) return nullptr;
    if (c.num_streams == 1) return c.stream[0];
    const uint64_t id = s->stream_counter % c.num_streams;
    s->stream_counter++;
    return c.stream[id];
}

void record_stream_event(PfSolveApplication* app, cudaStream_t stream)
{
    PfSolveConfiguration& c = app->configuration;
    AppState* s = st(app);
    if (c.num_streams > 1 && s->events) {
        const uint64_t id = (s->stream_counter + c.num_streams - 1) % c.num_streams;
        cudaEventRecord(s->events[id], stream);
    }
}

struct Resolved {
    void* bands;
    void* rhs;
    int64_t offM, offV, offS, iS, oS;
    int64_t iz0, iz1, oz0, oz1;
    double scaleC;
    int64_t batch;
};

PfSolveResult resolve(PfSolveApplication* app, const PfSolveLaunchParams* lp, Resolved& r)
{
    PfSolveConfiguration& c = app->configuration;
    const int64_t bm = c.jw_control_bitmask;
    if (lp && lp->batchSize > 0) c.size[1] = lp->batchSize;  // persists, as in the reference
    r.bands = (lp && lp->buffer) ? lp->buffer[0] : (c.buffer ? c.buffer[0] : nullptr);
    r.rhs = (lp && lp->outputBuffer) ? lp->outputBuffer[0] : (c.outputBuffer ? c.outputBuffer[0] : nullptr);
    if (!r.rhs) return PFSOLVE_ERROR_EMPTY_outputBuffer;
    auto pick = [&](int64_t bit, int64_t cfgv, uint64_t runv) -> int64_t {
        return (bm & bit) ? (lp ? (int64_t)runv : 0) : cfgv;
    };
    r.offM = pick(RUNTIME_OFFSETM, c.offsetM, lp ? lp->offsetM : 0);
    r.offV = pick(RUNTIME_OFFSETV, c.offsetV, lp ? lp->offsetV : 0);
    r.offS = pick(RUNTIME_OFFSETSOLUTION, c.offsetSolution, lp ? lp->offsetSolution : 0);
    r.iS = pick(RUNTIME_INPUTBUFFERSTRIDE, (int64_t)c.inputBufferStride[0], lp ? lp->inputBufferStride : 0);
    r.oS = pick(RUNTIME_OUTPUTBUFFERSTRIDE, (int64_t)c.outputBufferStride[0], lp ? lp->outputBufferStride : 0);
    const bool rtIZ = (bm & RUNTIME_INPUTZEROPAD) != 0, rtOZ = (bm & RUNTIME_OUTPUTZEROPAD) != 0;
    keep_window(rtIZ, rtIZ ? (lp ? (int64_t)lp->inputZeropad[0] : 0) : c.inputZeropad[0],
                rtIZ ? (lp ? (int64_t)lp->inputZeropad[1] : 0) : c.inputZeropad[1], r.iz0, r.iz1);
    keep_window(rtOZ, rtOZ ? (lp ? (int64_t)lp->outputZeropad[0] : 0) : c.outputZeropad[0],
                rtOZ ? (lp ? (int64_t)lp->outputZeropad[1] : 0) : c.outputZeropad[1], r.oz0, r.oz1);
    r.scaleC = (bm & RUNTIME_SCALEC) ? (lp ? (double)lp->scaleC : 0.0) : c.scaleC;
    r.batch = (int64_t)c.size[1] * (int64_t)(c.size[2] ? c.size[2] : 1);
    return PFSOLVE_SUCCESS;
}

void fill_operator_common(AppState* s, const PfSolveConfiguration& c, JwOperator& op)
{
    memset(&op, 0, sizeof(op));
    op.M = c.M_size;
    set_band_order(c.M_size, op);
    op.scaleC = 1.0;
    op.refine_sweeps = s->refine_sweeps;
    op.bands32 = prec_f32_storage(s->prec) ? 1 : 0;
}

// Tensor maps of recent launches (encoding is host work; steady-state
// launches repeat the same buffers).
struct MapCacheEntry {
    const void* v;  // the stream or cluster variant the maps were encoded for
    JwIO io;
    CUtensorMap in, out;
    bool valid;
};
thread_local MapCacheEntry g_map_cache[8];
thread_local unsigned g_map_next = 0;

bool same_io(const JwIO& a, const JwIO& b)
{
    return a.in == b.in && a.out == b.out && a.in_off == b.in_off && a.in_stride == b.in_stride &&
           a.out_off == b.out_off && a.out_stride == b.out_stride && a.nsys == b.nsys && a.M == b.M;
}

const MapCacheEntry* row_maps(const void* key, int R, int LIN, int LOUT, int IB, int IBO, const JwIO& io, int es = 8)
{
    for (const MapCacheEntry& e : g_map_cache)
        if (e.valid && e.v == key && same_io(e.io, io)) return &e;
    MapCacheEntry& e = g_map_cache[g_map_next++ % 8];
    e.valid = false;
    if (!encode_row_maps(R, LIN, LOUT, IB, IBO, io, &e.in, &e.out, es)) return nullptr;
    e.v = key;
    e.io = io;
    e.valid = true;
    return &e;
}

const MapCacheEntry* stream_maps(const StreamVariant* v, const JwIO& io)
{
    return row_maps(v, v->R, v->LIN, v->LOUT, v->IB, v->IBO, io, prec_f32_storage(v->PREC) ? 4 : 8);
}

// Long systems: the cluster kernel, under the streaming kernel's buffer rules.
PfSolveResult launch_cluster(AppState* s, const JwOperator& op, const JwIO& io, cudaStream_t stream)
{
    const ClusterVariant* v = s->cluster_v;
    if (io.accumulate || io.oz0 > 0 || io.oz1 < io.M) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    const MapCacheEntry* e = row_maps(v, v->R, LAY_REAL, LAY_REAL, v->IB, v->IBO, io);
    if (!e) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    const int clusters = (int)std::max<int64_t>(1, std::min<int64_t>(io.nsys, s->cluster_max));
    const cudaError_t err = v->launch(clusters, v->smem_bytes, stream, &e->in, &e->out, op, io);
    note_launch(true);
    record_launch(PFSOLVE_KERNEL_CLUSTER, v->R, v->W * v->C, 1, v->KL, v->KU, v->SV, LAY_REAL, LAY_REAL, 0, PREC_F64,
                  0, (int64_t)clusters * v->C);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    }
    return PFSOLVE_SUCCESS;
}

// Long systems: the two-pass kernel, under the streaming kernel's buffer rules.
PfSolveResult launch_long(AppState* s, const JwOperator& op, const JwIO& io, cudaStream_t stream)
{
    const LongVariant* v = s->long_v;
    bool single = s->long_single;
    int grid = s->long_grid;
    if (io.accumulate || io.oz0 > 0 || io.oz1 < io.M || io.nsys > s->long_batch)
        return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    JwIO mio = io;  // the maps cover the whole chunks of R rows
    mio.M = (io.M / v->R) * v->R;
    const MapCacheEntry* e = row_maps(v, v->R, LAY_REAL, LAY_REAL, v->IB, v->IBO, mio);
    // Rows no tensor map can describe (stride or offset not a multiple of 16
    // bytes): the single pass moves them with plain loads and stores (a
    // two-pass plan's fallback, when it has one, shares its records).
    static const CUtensorMap kNoMap = {};
    JwIO lio = io;
    if (!e) {
        if (!single) {
            if (!s->long_v_fb) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
            v = s->long_v_fb;
            grid = s->long_grid_fb;
            single = true;
        }
        lio.plain = 1;
    }
    const CUtensorMap* tin = e ? &e->in : &kNoMap;
    const CUtensorMap* tout = e ? &e->out : &kNoMap;
    double* cst = s->long_red + (size_t)s->long_batch * s->long_NS * 8;
    double* tab = cst + (size_t)s->long_NS * 8;
    if (++s->long_epoch == 0) s->long_epoch = 1;  // 0 is the flags' initial value
    const cudaError_t err = v->launch(grid, stream, tin, tout, op, lio, s->long_red, cst, tab, s->long_NS,
                                      s->long_flags, s->long_epoch, single);
    note_launch(true);
    record_launch(PFSOLVE_KERNEL_LONG, v->R, v->W, v->G, v->KL, v->KU, v->SV, LAY_REAL, LAY_REAL, 0, PREC_F64, 0,
                  grid);
    // the table passes, and for two passes the carry kernel (solves only) and pass 2
    g_launches.fetch_add((single ? 1 : (s->sv != SV_NONE ? 3 : 2)) + (s->sv == SV_TRI ? 1 : 0),
                         std::memory_order_relaxed);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    }
    return PFSOLVE_SUCCESS;
}

// Launch on the streaming variant when the plan has one and this launch's
// buffers allow it (no accumulation, full output window, TMA-encodable rows).
bool launch_stream(AppState* s, const JwOperator& op, const JwIO& io, cudaStream_t stream)
{
    const StreamVariant* v = s->stream_v;
    if (!v || io.accumulate || io.oz0 > 0 || io.oz1 < io.M) return false;
    // ALT: the launch counts systems (two per row set); the kernel, row sets
    JwIO rs = io;
    if (v->ALT) rs.nsys = io.nsys / 2;
    const MapCacheEntry* e = stream_maps(v, rs);
    if (!e) return false;
    const int64_t want = (rs.nsys + s->stream_G - 1) / s->stream_G;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(want, s->stream_max_blocks));
    rs.nbuf = s->stream_nbuf;
    v->launch(dim3((unsigned)grid), dim3(32 * v->W * s->stream_G), v->smem_bytes(s->stream_G, s->stream_nbuf), stream,
              &e->in, &e->out, op, rs);
    record_launch(PFSOLVE_KERNEL_STREAMING, v->R, v->W, s->stream_G, v->KL, v->KU, v->SV, v->LIN, v->LOUT, v->SCALE,
                  v->PREC, v->ALT, grid);
    return true;
}

PfSolveResult launch_jw_variant(AppState* s, const JwOperator& op, const JwIO& io, cudaStream_t stream)
{
    if (io.nsys <= 0) return PFSOLVE_SUCCESS;
    if (s->long_v) return launch_long(s, op, io, stream);
    if (s->cluster_v) return launch_cluster(s, op, io, stream);
    if (launch_stream(s, op, io, stream)) {
        g_launches.fetch_add(1, std::memory_order_relaxed);
        g_stream_launches.fetch_add(1, std::memory_order_relaxed);
        if (cudaPeekAtLastError() != cudaSuccess) {
            cudaGetLastError();
            return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
        }
        return PFSOLVE_SUCCESS;
    }
    if (!s->variant) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;  // streaming-only plan
    const int64_t want = (io.nsys + s->G - 1) / s->G;
    int64_t grid = std::max<int64_t>(1, std::min<int64_t>(want, s->max_blocks));
    // ALT: a group keeps one parity, so the system step (grid x groups) is even
    if (io.alt && (grid * s->G) % 2) grid = grid > 1 ? grid - 1 : 2;
    const size_t smem = s->variant->smem_bytes(s->W, s->G);
    s->variant->launch(dim3((unsigned)grid), dim3(32 * s->W * s->G), smem, stream, op, io, s->W);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    {
        const JwVariant* v = s->variant;
        record_launch(PFSOLVE_KERNEL_GROUP, v->R, s->W, s->G, v->KL, v->KU, v->SV, v->LIN, v->LOUT, v->SCALE, v->PREC,
                      io.alt, grid);
    }
    if (cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();
        return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    }
    return PFSOLVE_SUCCESS;
}

// Band offsets of step s of a K-step launch (pfSolve_JonesWorland.h:117-207 for
// the matvec operand, :269-353 for the solve operand, with M_size = M_s).
void step_layout(const PfSolveConfiguration& c, int s, int K, JwStepDesc& d)
{
    const int ub = c.upperBanded, jwt = c.jw_type % 10;
    const int64_t Ms = ub ? c.M_size - s : c.M_size + s;
    d.M = Ms;
    d.off_md = d.off_mo = d.off_sl = d.off_su = 0;
    d.diag = 0;
    if (ub == 2) {
        d.diag = 1;
        d.off_md = Ms;
        d.off_sl = 0;
        d.off_su = 2 * Ms;
        return;
    }
    if (jwt != 2) {
        if (ub == 1) {
            d.diag = s == 0;
            d.off_md = 0;
            d.off_mo = s == 0 ? Ms : 0;
        } else {
            d.diag = s == K - 1;
            d.off_md = Ms;
            d.off_mo = 0;
        }
    }
    if (jwt != 1) {
        if (ub == 1) d.off_sl = s == 0 ? 2 * Ms : Ms;
        else d.off_su = s == K - 1 ? 2 * Ms : Ms;
    }
}

PfSolveResult append_steps(PfSolveApplication* app, const PfSolveLaunchParams* lp, const Resolved& r,
                           cudaStream_t stream)
{
    AppState* s = st(app);
    const PfSolveConfiguration& c = app->configuration;
    JwSteps S;
    memset(&S, 0, sizeof(S));
    S.K = s->K;
    S.perm = 1;
    S.scaleC = r.scaleC;
    S.M_in = c.M_size;
    for (int k = 0; k < s->K; ++k) {
        JwStepDesc& d = S.st[k];
        void* b = r.bands;
        if (s->steps_nbuf > 1) {
            void** arr = (lp && lp->buffer) ? lp->buffer : c.buffer;
            b = arr ? arr[k] : nullptr;
        }
        if (!b) return PFSOLVE_ERROR_EMPTY_buffer;
        d.bands = static_cast<const double*>(b);
        step_layout(c, k, s->K, d);
        d.perm_r = s->steps_r;
        d.perm_m = d.M % d.perm_r;
        d.perm_ceil = (d.M + d.perm_r - 1) / d.perm_r;
        d.perm_floor = d.M / d.perm_r;
    }
    S.M_out = S.st[s->K - 1].M;
    JwIO io;
    memset(&io, 0, sizeof(io));
    io.in = static_cast<const double*>(r.rhs);
    io.out = static_cast<double*>(r.rhs);
    io.in_off = io.out_off = r.offS;
    io.in_stride = io.out_stride = r.oS;
    io.iz0 = r.iz0; io.iz1 = r.iz1; io.oz0 = r.oz0; io.oz1 = r.oz1;
    io.nsys = r.batch;
    io.M = std::max(S.M_in, S.M_out);
    if (io.nsys <= 0) return PFSOLVE_SUCCESS;
    CUtensorMap tin, tout;
    if (s->seq_v && io.oz0 <= 0 && io.oz1 >= S.M_out &&
        encode_seq_maps(io, S.M_in, S.M_out, s->seq_v->CH, &tin, &tout)) {
        // 32 systems per warp; warps per CTA so that every SM's warps finish
        // their blocks in the same number of rounds
        const int64_t nblk = (io.nsys + 31) / 32;
        const int64_t cap = (int64_t)s->num_sms * s->seq_NW;
        const int64_t rounds = (nblk + cap - 1) / cap;
        const int nw = (int)std::max<int64_t>(1, (nblk + (int64_t)s->num_sms * rounds - 1) / ((int64_t)s->num_sms * rounds));
        const int64_t grid = std::min<int64_t>(s->num_sms, (nblk + nw - 1) / nw);
        const int64_t Mtab = c.upperBanded ? S.M_in : S.M_out;
        s->seq_v->launch(dim3((unsigned)grid), dim3(32 * nw), seq_steps_smem_bytes(S.K, Mtab, nw, s->seq_v->CH), stream,
                         &tin, &tout,
                         S, io);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        record_launch(PFSOLVE_KERNEL_STEPS_SWEEP, 0, 0, nw, c.upperBanded == 0 ? 1 : 0, c.upperBanded == 1 ? 1 : 0,
                      s->seq_v->SV ? (c.upperBanded ? SV_LOWER : SV_UPPER) : SV_NONE, LAY_REAL, LAY_REAL, 0,
                      PREC_F64, 0, grid);
        g_stream_launches.fetch_add(1, std::memory_order_relaxed);
        if (cudaPeekAtLastError() != cudaSuccess) {
            cudaGetLastError();
            return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
        }
        return PFSOLVE_SUCCESS;
    }
    const StepsVariant* v = s->steps_v;
    if (!v) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;  // sweep-only plan, buffers it cannot take
    const int64_t want = (io.nsys + s->steps_G - 1) / s->steps_G;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(want, s->steps_max_blocks));
    v->launch(dim3((unsigned)grid), dim3(32 * s->steps_W * s->steps_G), v->smem_bytes(s->K, s->steps_W, s->steps_G),
              stream, S, io, s->steps_W);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    record_launch(PFSOLVE_KERNEL_STEPS, v->R, s->steps_W, s->steps_G, v->KL, v->KU, v->SV, LAY_REAL, LAY_REAL, 0,
                  PREC_F64, 0, grid);
    if (cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();
        return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    }
    return PFSOLVE_SUCCESS;
}

PfSolveResult append_jw(PfSolveApplication* app, const PfSolveLaunchParams* lp, cudaStream_t stream)
{
    AppState* s = st(app);
    const PfSolveConfiguration& c = app->configuration;
    Resolved r;
    PfSolveResult res = resolve(app, lp, r);
    if (res != PFSOLVE_SUCCESS) return res;
    if (!r.bands) return PFSOLVE_ERROR_EMPTY_buffer;
    if (s->K > 1) return append_steps(app, lp, r, stream);
    JwLayout L;
    if (s->alt) {
        PfSolveConfiguration ca = c;  // ALT: bands R T entries apart
        ca.M_size = s->alt_R * s->alt_T;
        jw_layout(ca, false, false, 0, 0, L);
    } else {
        jw_layout(c, (c.jw_control_bitmask & RUNTIME_OFFSETM) != 0, (c.jw_control_bitmask & RUNTIME_OFFSETV) != 0,
                  r.offM, r.offV, L);
    }
    JwOperator op;
    fill_operator_common(s, c, op);
    op.bands = static_cast<const double*>(r.bands);
    op.off_md = L.off_md;
    op.off_mo = L.off_mo;
    op.off_sl = L.off_sl;
    op.off_su = L.off_su;
    op.mvj = L.mvj;
    op.scaleC = r.scaleC;
    JwIO io;
    memset(&io, 0, sizeof(io));
    io.in = static_cast<const double*>(r.rhs);
    io.out = static_cast<double*>(r.rhs);
    io.in_off = io.out_off = r.offS;
    io.in_stride = io.out_stride = r.oS;  // the JW kernel addresses rows with outputBufferStride
    io.iz0 = r.iz0; io.iz1 = r.iz1; io.oz0 = r.oz0; io.oz1 = r.oz1;
    io.nsys = r.batch;
    io.M = c.M_size;
    if (s->alt) {
        op.alt = 1;
        op.alt_T = s->alt_T;
        op.alt_R = s->alt_R;
        io.alt = 1;
        io.nsys = 2 * r.batch;  // system 2y + h: the parity-h rows of right-hand side y
    }
    return launch_jw_variant(s, op, io, stream);
}

PfSolveResult append_dgbmv(PfSolveApplication* app, const PfSolveLaunchParams* lp, cudaStream_t stream)
{
    AppState* s = st(app);
    const PfSolveConfiguration& c = app->configuration;
    Resolved r;
    PfSolveResult res = resolve(app, lp, r);
    if (res != PFSOLVE_SUCCESS) return res;
    if (!r.bands) return PFSOLVE_ERROR_EMPTY_buffer;
    if (s->variant) {
        JwOperator op;
        fill_operator_common(s, c, op);
        op.bands = static_cast<const double*>(r.bands);  // unused by MVJ_NONE
        op.mvj = MVJ_NONE;
        op.dgbmv = static_cast<const double*>(r.bands);
        op.dg_off = r.offM;
        op.dg_lda = c.LDA;
        op.dg_ku = c.KU;
        op.dg_skip = s->dg_skip;
        JwIO io;
        memset(&io, 0, sizeof(io));
        io.in = static_cast<const double*>(r.rhs);
        io.out = static_cast<double*>(r.rhs);
        io.in_off = io.out_off = r.offS;
        io.in_stride = io.out_stride = r.oS;
        io.iz0 = r.iz0; io.iz1 = r.iz1; io.oz0 = r.oz0; io.oz1 = r.oz1;
        io.nsys = r.batch;
        io.M = c.M_size;
        return launch_jw_variant(s, op, io, stream);
    }
    if (s->prec && !prec_f32_storage(s->prec)) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    DgbmvArgs a;
    a.f32 = prec_f32_storage(s->prec) ? 1 : 0;
    a.A = static_cast<const double*>(r.bands);
    a.x = static_cast<double*>(r.rhs);
    a.M = c.M_size;
    a.nsys = r.batch;
    a.off_A = r.offM;
    a.off_x = r.offS;
    a.stride = r.oS;
    a.lda = c.LDA;
    a.ku = c.KU;
    a.skip = s->dg_skip;
    a.iz0 = r.iz0; a.iz1 = r.iz1; a.oz0 = r.oz0; a.oz1 = r.oz1;
    launch_dgbmv_generic(a, stream, s->num_sms);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    record_launch(PFSOLVE_KERNEL_DGBMV, 0, 0, 0, c.LDA - 1 - c.KU, c.KU, SV_NONE, LAY_REAL, LAY_REAL, 0, s->prec, 0, 0);
    if (cudaPeekAtLastError() != cudaSuccess) { cudaGetLastError(); return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL; }
    return PFSOLVE_SUCCESS;
}

PfSolveResult append_block(PfSolveApplication* app, const PfSolveLaunchParams* lp, cudaStream_t stream)
{
    AppState* s = st(app);
    const PfSolveConfiguration& c = app->configuration;
    Resolved r;
    PfSolveResult res = resolve(app, lp, r);
    if (res != PFSOLVE_SUCCESS) return res;
    if (!r.bands) return PFSOLVE_ERROR_EMPTY_buffer;
    BlockArgs a;
    a.f32 = prec_f32_storage(s->prec) ? 1 : 0;
    a.in = static_cast<const double*>(r.bands);
    a.out = static_cast<double*>(r.rhs);
    a.size0 = (int64_t)c.size[0];
    a.size1 = r.batch;
    a.in_off = r.offM;
    a.in_stride = r.iS;
    a.out_off = r.offS;
    a.out_stride = r.oS;
    a.iz0 = r.iz0; a.iz1 = r.iz1; a.oz0 = r.oz0; a.oz1 = r.oz1;
    a.layout = c.block % 10;
    a.accumulate = ((c.block / 10) % 10) == 2;
    a.scale_kind = c.block / 100;
    a.lshift = c.lshift;
    a.s = r.scaleC;
    a.skip_read = (a.scale_kind == 1) && !(c.jw_control_bitmask & RUNTIME_SCALEC) && c.scaleC == 0.0;
    launch_block(a, stream, s->num_sms);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    record_launch(PFSOLVE_KERNEL_BLOCK, 0, 0, 0, 0, 0, SV_NONE, 0, 0, a.scale_kind != 0, s->prec, 0, 0);
    if (cudaPeekAtLastError() != cudaSuccess) { cudaGetLastError(); return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL; }
    return PFSOLVE_SUCCESS;
}

// The DCT step: rows from `buffer` (launch-time buffer first) at the input
// stride, results to `outputBuffer`, or in place when there is none.  Runtime
// input / output strides and offsets follow the same RUNTIME_* bits as the
// other applications (offsetM: input rows, offsetSolution: output rows).
PfSolveResult append_dct(PfSolveApplication* app, const PfSolveLaunchParams* lp, cudaStream_t stream)
{
    AppState* s = st(app);
    PfSolveConfiguration& c = app->configuration;
    const int64_t bm = c.jw_control_bitmask;
    if (lp && lp->batchSize > 0) c.size[1] = lp->batchSize;  // persists, as in the reference
    void* in = (lp && lp->buffer) ? lp->buffer[0] : (c.buffer ? c.buffer[0] : nullptr);
    void* out = (lp && lp->outputBuffer) ? lp->outputBuffer[0] : (c.outputBuffer ? c.outputBuffer[0] : nullptr);
    if (!in) return PFSOLVE_ERROR_EMPTY_buffer;
    if (!out) out = in;
    auto pick = [&](int64_t bit, int64_t cfgv, uint64_t runv) -> int64_t {
        return (bm & bit) ? (lp ? (int64_t)runv : 0) : cfgv;
    };
    const int64_t N = (int64_t)c.size[0];
    DctIO io;
    io.in = static_cast<const double*>(in);
    io.out = static_cast<double*>(out);
    io.in_off = pick(RUNTIME_OFFSETM, c.offsetM, lp ? lp->offsetM : 0);
    io.out_off = pick(RUNTIME_OFFSETSOLUTION, c.offsetSolution, lp ? lp->offsetSolution : 0);
    io.in_stride = pick(RUNTIME_INPUTBUFFERSTRIDE, (int64_t)c.inputBufferStride[0], lp ? lp->inputBufferStride : 0);
    io.out_stride =
        pick(RUNTIME_OUTPUTBUFFERSTRIDE, (int64_t)c.outputBufferStride[0], lp ? lp->outputBufferStride : 0);
    if (io.in_stride == 0) io.in_stride = N;
    if (io.out_stride == 0) io.out_stride = N;
    if (io.in_stride < N || io.out_stride < N || io.in_off < 0 || io.out_off < 0) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    io.nsys = (int64_t)c.size[1] * (int64_t)(c.size[2] ? c.size[2] : 1);
    if (io.nsys <= 0) return PFSOLVE_SUCCESS;
    // in place needs each row's input and output at the same place
    if (out == in && (io.in_off != io.out_off || io.in_stride != io.out_stride)) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    const double2* tw = s->dct_tables;
    const double2* pt = s->dct_tables + N;
    const cudaError_t e = dct_launch(s->dct_logn, (int)c.performDCT, io, tw, pt, s->num_sms, stream);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    record_launch(PFSOLVE_KERNEL_DCT, 0, 0, 0, 0, 0, SV_NONE, 0, 0, 0, PREC_F64, 0, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    }
    return PFSOLVE_SUCCESS;
}

}  // namespace

extern "C" {

const char* getPfSolveErrorString(PfSolveResult result)
{
    // every code of the header's PfSolveResult, each with its own name
    static const struct {
        PfSolveResult code;
        const char* name;
    } kNames[] = {
        {PFSOLVE_SUCCESS, "PFSOLVE_SUCCESS"},
        {PFSOLVE_ERROR_MALLOC_FAILED, "PFSOLVE_ERROR_MALLOC_FAILED"},
        {PFSOLVE_ERROR_INSUFFICIENT_CODE_BUFFER, "PFSOLVE_ERROR_INSUFFICIENT_CODE_BUFFER"},
        {PFSOLVE_ERROR_INSUFFICIENT_TEMP_BUFFER, "PFSOLVE_ERROR_INSUFFICIENT_TEMP_BUFFER"},
        {PFSOLVE_ERROR_PLAN_NOT_INITIALIZED, "PFSOLVE_ERROR_PLAN_NOT_INITIALIZED"},
        {PFSOLVE_ERROR_NULL_TEMP_PASSED, "PFSOLVE_ERROR_NULL_TEMP_PASSED"},
        {PFSOLVE_ERROR_MATH_FAILED, "PFSOLVE_ERROR_MATH_FAILED"},
        {PFSOLVE_ERROR_INVALID_PHYSICAL_DEVICE, "PFSOLVE_ERROR_INVALID_PHYSICAL_DEVICE"},
        {PFSOLVE_ERROR_INVALID_DEVICE, "PFSOLVE_ERROR_INVALID_DEVICE"},
        {PFSOLVE_ERROR_INVALID_QUEUE, "PFSOLVE_ERROR_INVALID_QUEUE"},
        {PFSOLVE_ERROR_INVALID_COMMAND_POOL, "PFSOLVE_ERROR_INVALID_COMMAND_POOL"},
        {PFSOLVE_ERROR_INVALID_FENCE, "PFSOLVE_ERROR_INVALID_FENCE"},
        {PFSOLVE_ERROR_ONLY_FORWARD_FFT_INITIALIZED, "PFSOLVE_ERROR_ONLY_FORWARD_FFT_INITIALIZED"},
        {PFSOLVE_ERROR_ONLY_INVERSE_FFT_INITIALIZED, "PFSOLVE_ERROR_ONLY_INVERSE_FFT_INITIALIZED"},
        {PFSOLVE_ERROR_INVALID_CONTEXT, "PFSOLVE_ERROR_INVALID_CONTEXT"},
        {PFSOLVE_ERROR_INVALID_PLATFORM, "PFSOLVE_ERROR_INVALID_PLATFORM"},
        {PFSOLVE_ERROR_ENABLED_saveApplicationToString, "PFSOLVE_ERROR_ENABLED_saveApplicationToString"},
        {PFSOLVE_ERROR_EMPTY_FILE, "PFSOLVE_ERROR_EMPTY_FILE"},
        {PFSOLVE_ERROR_EMPTY_FFTdim, "PFSOLVE_ERROR_EMPTY_FFTdim"},
        {PFSOLVE_ERROR_EMPTY_size, "PFSOLVE_ERROR_EMPTY_size"},
        {PFSOLVE_ERROR_EMPTY_bufferSize, "PFSOLVE_ERROR_EMPTY_bufferSize"},
        {PFSOLVE_ERROR_EMPTY_buffer, "PFSOLVE_ERROR_EMPTY_buffer"},
        {PFSOLVE_ERROR_EMPTY_tempBufferSize, "PFSOLVE_ERROR_EMPTY_tempBufferSize"},
        {PFSOLVE_ERROR_EMPTY_tempBuffer, "PFSOLVE_ERROR_EMPTY_tempBuffer"},
        {PFSOLVE_ERROR_EMPTY_inputBufferSize, "PFSOLVE_ERROR_EMPTY_inputBufferSize"},
        {PFSOLVE_ERROR_EMPTY_inputBuffer, "PFSOLVE_ERROR_EMPTY_inputBuffer"},
        {PFSOLVE_ERROR_EMPTY_outputBufferSize, "PFSOLVE_ERROR_EMPTY_outputBufferSize"},
        {PFSOLVE_ERROR_EMPTY_outputBuffer, "PFSOLVE_ERROR_EMPTY_outputBuffer"},
        {PFSOLVE_ERROR_EMPTY_kernelSize, "PFSOLVE_ERROR_EMPTY_kernelSize"},
        {PFSOLVE_ERROR_EMPTY_kernel, "PFSOLVE_ERROR_EMPTY_kernel"},
        {PFSOLVE_ERROR_EMPTY_applicationString, "PFSOLVE_ERROR_EMPTY_applicationString"},
        {PFSOLVE_ERROR_EMPTY_useCustomBluesteinPaddingPattern_arrays, "PFSOLVE_ERROR_EMPTY_useCustomBluesteinPaddingPattern_arrays"},
        {PFSOLVE_ERROR_UNSUPPORTED_RADIX, "PFSOLVE_ERROR_UNSUPPORTED_RADIX"},
        {PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH, "PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH"},
        {PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_R2C, "PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_R2C"},
        {PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_DCT, "PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_DCT"},
        {PFSOLVE_ERROR_UNSUPPORTED_FFT_OMIT, "PFSOLVE_ERROR_UNSUPPORTED_FFT_OMIT"},
        {PFSOLVE_ERROR_FAILED_TO_ALLOCATE, "PFSOLVE_ERROR_FAILED_TO_ALLOCATE"},
        {PFSOLVE_ERROR_FAILED_TO_MAP_MEMORY, "PFSOLVE_ERROR_FAILED_TO_MAP_MEMORY"},
        {PFSOLVE_ERROR_FAILED_TO_ALLOCATE_COMMAND_BUFFERS, "PFSOLVE_ERROR_FAILED_TO_ALLOCATE_COMMAND_BUFFERS"},
        {PFSOLVE_ERROR_FAILED_TO_BEGIN_COMMAND_BUFFER, "PFSOLVE_ERROR_FAILED_TO_BEGIN_COMMAND_BUFFER"},
        {PFSOLVE_ERROR_FAILED_TO_END_COMMAND_BUFFER, "PFSOLVE_ERROR_FAILED_TO_END_COMMAND_BUFFER"},
        {PFSOLVE_ERROR_FAILED_TO_SUBMIT_QUEUE, "PFSOLVE_ERROR_FAILED_TO_SUBMIT_QUEUE"},
        {PFSOLVE_ERROR_FAILED_TO_WAIT_FOR_FENCES, "PFSOLVE_ERROR_FAILED_TO_WAIT_FOR_FENCES"},
        {PFSOLVE_ERROR_FAILED_TO_RESET_FENCES, "PFSOLVE_ERROR_FAILED_TO_RESET_FENCES"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_DESCRIPTOR_POOL, "PFSOLVE_ERROR_FAILED_TO_CREATE_DESCRIPTOR_POOL"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_DESCRIPTOR_SET_LAYOUT, "PFSOLVE_ERROR_FAILED_TO_CREATE_DESCRIPTOR_SET_LAYOUT"},
        {PFSOLVE_ERROR_FAILED_TO_ALLOCATE_DESCRIPTOR_SETS, "PFSOLVE_ERROR_FAILED_TO_ALLOCATE_DESCRIPTOR_SETS"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_PIPELINE_LAYOUT, "PFSOLVE_ERROR_FAILED_TO_CREATE_PIPELINE_LAYOUT"},
        {PFSOLVE_ERROR_FAILED_SHADER_PREPROCESS, "PFSOLVE_ERROR_FAILED_SHADER_PREPROCESS"},
        {PFSOLVE_ERROR_FAILED_SHADER_PARSE, "PFSOLVE_ERROR_FAILED_SHADER_PARSE"},
        {PFSOLVE_ERROR_FAILED_SHADER_LINK, "PFSOLVE_ERROR_FAILED_SHADER_LINK"},
        {PFSOLVE_ERROR_FAILED_SPIRV_GENERATE, "PFSOLVE_ERROR_FAILED_SPIRV_GENERATE"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_SHADER_MODULE, "PFSOLVE_ERROR_FAILED_TO_CREATE_SHADER_MODULE"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_INSTANCE, "PFSOLVE_ERROR_FAILED_TO_CREATE_INSTANCE"},
        {PFSOLVE_ERROR_FAILED_TO_SETUP_DEBUG_MESSENGER, "PFSOLVE_ERROR_FAILED_TO_SETUP_DEBUG_MESSENGER"},
        {PFSOLVE_ERROR_FAILED_TO_FIND_PHYSICAL_DEVICE, "PFSOLVE_ERROR_FAILED_TO_FIND_PHYSICAL_DEVICE"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_DEVICE, "PFSOLVE_ERROR_FAILED_TO_CREATE_DEVICE"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_FENCE, "PFSOLVE_ERROR_FAILED_TO_CREATE_FENCE"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_COMMAND_POOL, "PFSOLVE_ERROR_FAILED_TO_CREATE_COMMAND_POOL"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_BUFFER, "PFSOLVE_ERROR_FAILED_TO_CREATE_BUFFER"},
        {PFSOLVE_ERROR_FAILED_TO_ALLOCATE_MEMORY, "PFSOLVE_ERROR_FAILED_TO_ALLOCATE_MEMORY"},
        {PFSOLVE_ERROR_FAILED_TO_BIND_BUFFER_MEMORY, "PFSOLVE_ERROR_FAILED_TO_BIND_BUFFER_MEMORY"},
        {PFSOLVE_ERROR_FAILED_TO_FIND_MEMORY, "PFSOLVE_ERROR_FAILED_TO_FIND_MEMORY"},
        {PFSOLVE_ERROR_FAILED_TO_SYNCHRONIZE, "PFSOLVE_ERROR_FAILED_TO_SYNCHRONIZE"},
        {PFSOLVE_ERROR_FAILED_TO_COPY, "PFSOLVE_ERROR_FAILED_TO_COPY"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_PROGRAM, "PFSOLVE_ERROR_FAILED_TO_CREATE_PROGRAM"},
        {PFSOLVE_ERROR_FAILED_TO_COMPILE_PROGRAM, "PFSOLVE_ERROR_FAILED_TO_COMPILE_PROGRAM"},
        {PFSOLVE_ERROR_FAILED_TO_GET_CODE_SIZE, "PFSOLVE_ERROR_FAILED_TO_GET_CODE_SIZE"},
        {PFSOLVE_ERROR_FAILED_TO_GET_CODE, "PFSOLVE_ERROR_FAILED_TO_GET_CODE"},
        {PFSOLVE_ERROR_FAILED_TO_DESTROY_PROGRAM, "PFSOLVE_ERROR_FAILED_TO_DESTROY_PROGRAM"},
        {PFSOLVE_ERROR_FAILED_TO_LOAD_MODULE, "PFSOLVE_ERROR_FAILED_TO_LOAD_MODULE"},
        {PFSOLVE_ERROR_FAILED_TO_GET_FUNCTION, "PFSOLVE_ERROR_FAILED_TO_GET_FUNCTION"},
        {PFSOLVE_ERROR_FAILED_TO_SET_DYNAMIC_SHARED_MEMORY, "PFSOLVE_ERROR_FAILED_TO_SET_DYNAMIC_SHARED_MEMORY"},
        {PFSOLVE_ERROR_FAILED_TO_MODULE_GET_GLOBAL, "PFSOLVE_ERROR_FAILED_TO_MODULE_GET_GLOBAL"},
        {PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL, "PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL"},
        {PFSOLVE_ERROR_FAILED_TO_EVENT_RECORD, "PFSOLVE_ERROR_FAILED_TO_EVENT_RECORD"},
        {PFSOLVE_ERROR_FAILED_TO_ADD_NAME_EXPRESSION, "PFSOLVE_ERROR_FAILED_TO_ADD_NAME_EXPRESSION"},
        {PFSOLVE_ERROR_FAILED_TO_INITIALIZE, "PFSOLVE_ERROR_FAILED_TO_INITIALIZE"},
        {PFSOLVE_ERROR_FAILED_TO_SET_DEVICE_ID, "PFSOLVE_ERROR_FAILED_TO_SET_DEVICE_ID"},
        {PFSOLVE_ERROR_FAILED_TO_GET_DEVICE, "PFSOLVE_ERROR_FAILED_TO_GET_DEVICE"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_CONTEXT, "PFSOLVE_ERROR_FAILED_TO_CREATE_CONTEXT"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_PIPELINE, "PFSOLVE_ERROR_FAILED_TO_CREATE_PIPELINE"},
        {PFSOLVE_ERROR_FAILED_TO_SET_KERNEL_ARG, "PFSOLVE_ERROR_FAILED_TO_SET_KERNEL_ARG"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_COMMAND_QUEUE, "PFSOLVE_ERROR_FAILED_TO_CREATE_COMMAND_QUEUE"},
        {PFSOLVE_ERROR_FAILED_TO_RELEASE_COMMAND_QUEUE, "PFSOLVE_ERROR_FAILED_TO_RELEASE_COMMAND_QUEUE"},
        {PFSOLVE_ERROR_FAILED_TO_ENUMERATE_DEVICES, "PFSOLVE_ERROR_FAILED_TO_ENUMERATE_DEVICES"},
        {PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE, "PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_EVENT, "PFSOLVE_ERROR_FAILED_TO_CREATE_EVENT"},
        {PFSOLVE_ERROR_FAILED_TO_CREATE_COMMAND_LIST, "PFSOLVE_ERROR_FAILED_TO_CREATE_COMMAND_LIST"},
        {PFSOLVE_ERROR_FAILED_TO_DESTROY_COMMAND_LIST, "PFSOLVE_ERROR_FAILED_TO_DESTROY_COMMAND_LIST"},
        {PFSOLVE_ERROR_FAILED_TO_SUBMIT_BARRIER, "PFSOLVE_ERROR_FAILED_TO_SUBMIT_BARRIER"},
        {PFSOLVE_ERROR_UNSUPPORTED_COMBINATION, "PFSOLVE_ERROR_UNSUPPORTED_COMBINATION"},
        {PFSOLVE_ERROR_INVALID_ARGUMENT, "PFSOLVE_ERROR_INVALID_ARGUMENT"},
        {PFSOLVE_ERROR_CAPACITY, "PFSOLVE_ERROR_CAPACITY"},
        {PFSOLVE_ERROR_DEVICE_FAULT, "PFSOLVE_ERROR_DEVICE_FAULT"},
    };
    for (const auto& e : kNames)
        if (e.code == result) return e.name;
    return "PFSOLVE_ERROR_UNKNOWN";
}

// The reference's version function returns the literal 00102 (pfSolve.h:101-103),
// an octal literal whose value is 66.
int PfSolveGetVersion(void) { return 66; }

uint64_t PfSolveLaunchCount(void) { return g_launches.load(); }

uint64_t PfSolveStreamingLaunchCount(void) { return g_stream_launches.load(); }

PfSolveResult PfSolveGetLastLaunch(PfSolveLaunchInfo* info)
{
    if (!info) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    *info = g_last_launch;
    return PFSOLVE_SUCCESS;
}

PfSolveResult PfSolveGetShape(const PfSolveApplication* app, int* streaming, int* rowsPerThread, int* warpsPerSystem,
                              int* groupsPerCTA)
{
    if (!app || !app->internal) return PFSOLVE_ERROR_PLAN_NOT_INITIALIZED;
    const AppState* s = static_cast<const AppState*>(app->internal);
    if (s->seq_v) {
        if (streaming) *streaming = 4;
        if (rowsPerThread) *rowsPerThread = 0;
        if (warpsPerSystem) *warpsPerSystem = 0;
        if (groupsPerCTA) *groupsPerCTA = s->seq_NW;
        return PFSOLVE_SUCCESS;
    }
    if (s->steps_v) {
        if (streaming) *streaming = 3;
        if (rowsPerThread) *rowsPerThread = s->steps_v->R;
        if (warpsPerSystem) *warpsPerSystem = s->steps_W;
        if (groupsPerCTA) *groupsPerCTA = s->steps_G;
        return PFSOLVE_SUCCESS;
    }
    if (s->long_v) {
        if (streaming) *streaming = 5;
        if (rowsPerThread) *rowsPerThread = s->long_v->R;
        if (warpsPerSystem) *warpsPerSystem = s->long_v->W;
        if (groupsPerCTA) *groupsPerCTA = s->long_v->G;
        return PFSOLVE_SUCCESS;
    }
    if (s->cluster_v) {
        if (streaming) *streaming = 2;
        if (rowsPerThread) *rowsPerThread = s->cluster_v->R;
        if (warpsPerSystem) *warpsPerSystem = s->cluster_v->W * s->cluster_v->C;
        if (groupsPerCTA) *groupsPerCTA = 1;
        return PFSOLVE_SUCCESS;
    }
    const bool sm = s->stream_v != nullptr;
    if (streaming) *streaming = sm ? 1 : 0;
    if (rowsPerThread) *rowsPerThread = sm ? s->stream_v->R : s->R;
    if (warpsPerSystem) *warpsPerSystem = sm ? s->stream_v->W : s->W;
    if (groupsPerCTA) *groupsPerCTA = sm ? s->stream_G : s->G;
    return PFSOLVE_SUCCESS;
}

PfSolveResult initializePfSolve(PfSolveApplication* app, PfSolveConfiguration cfg)
{
    if (!app) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    memset(app, 0, sizeof(*app));
    app->configuration = cfg;
    PfSolveConfiguration& c = app->configuration;
    if (c.FFTdim != 1) return PFSOLVE_ERROR_EMPTY_FFTdim;
    if (!c.device) return PFSOLVE_ERROR_INVALID_DEVICE;
    if (c.size[0] == 0) return PFSOLVE_ERROR_EMPTY_size;
    if (c.size[1] == 0) c.size[1] = 1;
    if (c.size[2] == 0) c.size[2] = 1;
    if (c.M_size == 0) c.M_size = (int64_t)c.size[0];
    if (c.inputBufferStride[0] == 0) c.inputBufferStride[0] = c.size[0];
    if (c.outputBufferStride[0] == 0) c.outputBufferStride[0] = c.size[0];
    if (c.halfPrecision) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;

    AppState* s = new (std::nothrow) AppState();
    if (!s) return PFSOLVE_ERROR_MALLOC_FAILED;
    app->internal = s;
    s->device = *c.device;
    if (c.stagingBuffers != 0 && (c.stagingBuffers < 2 || c.stagingBuffers > kStMaxBuffers)) {
        deletePfSolve(app);
        return PFSOLVE_ERROR_INVALID_ARGUMENT;
    }
    s->nbuf_req = c.stagingBuffers;
    if (cudaSetDevice(s->device) != cudaSuccess) { deletePfSolve(app); return PFSOLVE_ERROR_INVALID_DEVICE; }
    if (cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess) {
        deletePfSolve(app);
        return PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE;
    }
    if (c.num_streams > 1) {
        if (!c.stream) { deletePfSolve(app); return PFSOLVE_ERROR_INVALID_ARGUMENT; }
        s->events = new (std::nothrow) cudaEvent_t[c.num_streams];
        if (!s->events) { deletePfSolve(app); return PFSOLVE_ERROR_MALLOC_FAILED; }
        for (uint64_t i = 0; i < c.num_streams; i++) {
            if (cudaEventCreateWithFlags(&s->events[i], cudaEventDisableTiming) != cudaSuccess) {
                deletePfSolve(app);
                return PFSOLVE_ERROR_FAILED_TO_EVENT_RECORD;
            }
        }
    }
    // Precision, in the reference's order (pfSolve_InitAPIParameters.h:148-245,
    // pfSolve_Plan_JonesWorland.h:244-264): double-double storage
    // (quadDoubleDoublePrecision) or arithmetic on FP64 storage
    // (quadDoubleDoublePrecisionDoubleMemory); FP64 (doublePrecision,
    // optionally with the FP32-solve refinement extension); FP64 arithmetic on
    // FP32 storage (doublePrecisionFloatMemory); else FP32 storage and
    // arithmetic, the reference's default.
    const bool ddmem = c.quadDoubleDoublePrecision != 0;
    const bool ddf64 = !ddmem && c.quadDoubleDoublePrecisionDoubleMemory != 0;
    const int dd_prec = ddmem ? 2 : (ddf64 ? 3 : 0);
    const int base_prec = dd_prec                        ? dd_prec
                          : c.doublePrecision            ? PREC_F64
                          : c.doublePrecisionFloatMemory ? PREC_F64_F32MEM
                                                         : PREC_F32;
    PfSolveResult r = PFSOLVE_SUCCESS;
    if (c.performDCT) {
        // the DCT step: rows of N = 2^p points, FP64
        s->kind = APP_DCT;
        const int64_t N = (int64_t)c.size[0];
        int logn = 0;
        while ((int64_t)1 << logn < N) ++logn;
        if (c.performDCT != 2 && c.performDCT != 3) r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        else if (c.FFTdim != 1 || N < 8 || N > 4096 || ((int64_t)1 << logn) != N)
            r = PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH_DCT;
        else if (base_prec != PREC_F64) r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        else if (dct_tables(N, &s->dct_tables) != cudaSuccess) {
            cudaGetLastError();
            s->dct_tables = nullptr;
            r = PFSOLVE_ERROR_FAILED_TO_ALLOCATE;
        } else {
            s->dct_logn = logn;
            s->prec = PREC_F64;
        }
    } else if (c.jw_type >= 10) {
        s->kind = APP_JW;
        if (c.mixedPrecisionRefinement < 0 || c.mixedPrecisionRefinement > 3) r = PFSOLVE_ERROR_INVALID_ARGUMENT;
        else if (c.mixedPrecisionRefinement && base_prec != PREC_F64) r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        else if (((c.jw_type / 100) % 10) == 1) r = plan_alt(s, c, base_prec);
        else if (c.upperBanded < 0 || c.upperBanded > 2) r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        else if (c.numConsecutiveJWIterations > 1) {
            s->prec = base_prec;
            r = plan_steps(s, c);
        }
        else if (c.M_size > kMaxRowsLong || c.M_size < 1) r = PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH;
        else {
            JwLayout L;
            if (!jw_layout(c, false, false, 0, 0, L)) r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
            else {
                s->mvj = L.mvj;
                s->sv = L.sv;
                s->prec = base_prec != PREC_F64 ? base_prec
                                                : ((c.mixedPrecisionRefinement > 0 && L.sv != SV_NONE) ? PREC_MIXED
                                                                                                       : PREC_F64);
                s->refine_sweeps = 1 + c.mixedPrecisionRefinement;
                s->KL = (L.mvj == MVJ_LOWER) ? 1 : 0;
                s->KU = (L.mvj == MVJ_UPPER) ? 1 : 0;
                s->R = pick_rows_per_thread(c.M_size, c.rowsPerThread);
                s->R_fixed = c.rowsPerThread != 0 && c.rowsPerThread != 32;
                s->R_req = c.rowsPerThread;
                s->no_stream = c.kernelPath == 1;
                s->cluster_only = c.kernelPath == 2;
                s->long_mode = c.kernelPath;
                s->plan_batch = (int64_t)c.size[1] * (int64_t)(c.size[2] ? c.size[2] : 1);
                r = finish_variant(s, c.M_size, LAY_REAL, LAY_REAL, 0);
            }
        }
    } else if (c.LDA > 0) {
        s->kind = APP_DGBMV;
        s->prec = base_prec;
        if (c.KU < 0 || c.KU >= c.LDA) r = PFSOLVE_ERROR_INVALID_ARGUMENT;
        else if (c.ALT_dgbmv && (c.LDA > 64 || dd_prec)) r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        else {
            // ALT_dgbmv (pfSolve_Plan_dgbmv.h:100, pfSolve_MatVecMul.h:390) drops band j
            // when (j % 2 == 1 - LDA % 2 and KL != 0) or (j % 2 == LDA % 2 and KU != 0),
            // KL and KU as configured
            if (c.ALT_dgbmv)
                for (int j = 0; j < c.LDA; ++j)
                    if (((j % 2) == 1 - (c.LDA % 2) && c.KL) || ((j % 2) == (c.LDA % 2) && c.KU))
                        s->dg_skip |= 1ull << j;
            const int kl = c.LDA - 1 - c.KU;
            if (dd_prec && !(kl == 1 && c.KU == 1)) r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
            else if (kl <= 2 && c.KU <= 2 && c.M_size <= kMaxRows) {
                s->KL = kl;
                s->KU = c.KU;
                s->sv = SV_NONE;
                s->mvj = MVJ_NONE;
                s->R = pick_rows_per_thread(c.M_size, c.rowsPerThread);
                if (s->R < 4) s->R = 4;
                s->R_req = c.rowsPerThread;
                s->no_stream = c.kernelPath == 1;
                r = finish_variant(s, c.M_size, LAY_REAL, LAY_REAL, 0);
            }
            // wider bands use the generic kernel (variant stays null)
        }
    } else if (c.block > 0) {
        s->kind = APP_BLOCK;
        const int bt = c.block % 10, acc = (c.block / 10) % 10, sk = c.block / 100;
        s->prec = base_prec;
        if (dd_prec) r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        else if (bt < 1 || bt > 7 || (acc != 0 && acc != 2) || sk > 4) r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        else if (acc == 2 && bt == 4) r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    } else {
        r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    }
    if (r != PFSOLVE_SUCCESS) {
        deletePfSolve(app);
        return r;
    }
    return PFSOLVE_SUCCESS;
}

PfSolveResult PfSolveAppend(PfSolveApplication* app, int inverse, PfSolveLaunchParams* launchParams)
{
    (void)inverse;
    if (!app || !app->internal) return PFSOLVE_ERROR_PLAN_NOT_INITIALIZED;
    AppState* s = st(app);
    cudaStream_t stream = pick_stream(app);
    PfSolveResult r;
    switch (s->kind) {
    case APP_JW: r = append_jw(app, launchParams, stream); break;
    case APP_DGBMV: r = append_dgbmv(app, launchParams, stream); break;
    case APP_BLOCK: r = append_block(app, launchParams, stream); break;
    case APP_DCT: r = append_dct(app, launchParams, stream); break;
    default: r = PFSOLVE_ERROR_PLAN_NOT_INITIALIZED;
    }
    if (r == PFSOLVE_SUCCESS) record_stream_event(app, stream);
    return r;
}

PfSolveResult PfSolveGetDeviceStatus(void)
{
    const unsigned v = stream_status_fetch_clear();
    if (v == ~0u) return PFSOLVE_ERROR_FAILED_TO_SYNCHRONIZE;
    return v ? PFSOLVE_ERROR_DEVICE_FAULT : PFSOLVE_SUCCESS;
}

PfSolveResult PfSolveSync(PfSolveApplication* app)
{
    if (!app || !app->internal) return PFSOLVE_ERROR_PLAN_NOT_INITIALIZED;
    AppState* s = st(app);
    const PfSolveConfiguration& c = app->configuration;
    if (c.num_streams > 1 && s->events) {
        for (uint64_t i = 0; i < c.num_streams; i++)
            if (cudaEventSynchronize(s->events[i]) != cudaSuccess) return PFSOLVE_ERROR_FAILED_TO_SYNCHRONIZE;
        s->stream_counter = 0;
    }
    return PFSOLVE_SUCCESS;
}

void deletePfSolve(PfSolveApplication* app)
{
    if (!app) return;
    AppState* s = st(app);
    if (s) {
        if (s->events) {
            for (uint64_t i = 0; i < app->configuration.num_streams; i++)
                if (s->events[i]) cudaEventDestroy(s->events[i]);
            delete[] s->events;
        }
        if (s->long_red) cudaFree(s->long_red);
        if (s->dct_tables) cudaFree(s->dct_tables);
        delete s;
    }
    app->internal = nullptr;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Fused chains: [dgbmv] -> JW -> [block] over the same systems, one kernel.
namespace {

bool trivial_window(int64_t lo, int64_t hi, int64_t M) { return lo <= 0 && hi >= M; }

PfSolveResult append_chain_fused(PfSolveApplication* dg, const PfSolveLaunchParams* dlp, PfSolveApplication* jw,
                                 const PfSolveLaunchParams* jlp, PfSolveApplication* bl,
                                 const PfSolveLaunchParams* blp, cudaStream_t stream)
{
    AppState* sj = st(jw);
    const PfSolveConfiguration& cj = jw->configuration;
    const int64_t M = cj.M_size;
    Resolved rj;
    PfSolveResult res = resolve(jw, jlp, rj);
    if (res != PFSOLVE_SUCCESS) return res;
    if (!rj.bands) return PFSOLVE_ERROR_EMPTY_buffer;
    JwLayout L;
    jw_layout(cj, (cj.jw_control_bitmask & RUNTIME_OFFSETM) != 0, (cj.jw_control_bitmask & RUNTIME_OFFSETV) != 0,
              rj.offM, rj.offV, L);
    int KL = (L.mvj == MVJ_LOWER) ? 1 : 0, KU = (L.mvj == MVJ_UPPER) ? 1 : 0;
    JwOperator op;
    fill_operator_common(sj, cj, op);
    op.bands = static_cast<const double*>(rj.bands);
    op.off_md = L.off_md; op.off_mo = L.off_mo; op.off_sl = L.off_sl; op.off_su = L.off_su;
    op.mvj = L.mvj;
    op.scaleC = rj.scaleC;
    JwIO io;
    memset(&io, 0, sizeof(io));
    io.M = M;
    io.in = static_cast<const double*>(rj.rhs);
    io.in_off = rj.offS;
    io.in_stride = rj.oS;
    io.iz0 = rj.iz0; io.iz1 = rj.iz1;
    io.oz0 = rj.oz0; io.oz1 = rj.oz1;
    io.out = static_cast<double*>(rj.rhs);
    io.out_off = rj.offS;
    io.out_stride = rj.oS;
    io.nsys = rj.batch;
    int LIN = LAY_REAL, LOUT = LAY_REAL, SCALE = 0;
    // with FP32 storage anywhere along the chain, one precision for all of it
    auto same_storage = [&](PfSolveApplication* a) {
        const int pa = st(a)->prec;
        return !(prec_f32_storage(pa) || prec_f32_storage(sj->prec)) || pa == sj->prec;
    };
    if ((dg && !same_storage(dg)) || (bl && !same_storage(bl))) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    if (dg) {
        const PfSolveConfiguration& cd = dg->configuration;
        Resolved rd;
        if ((res = resolve(dg, dlp, rd)) != PFSOLVE_SUCCESS) return res;
        if (cd.M_size != M || rd.rhs != rj.rhs || rd.offS != rj.offS || rd.oS != rj.oS || rd.batch != rj.batch)
            return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        if (!trivial_window(rd.oz0, rd.oz1, M) || !trivial_window(rj.iz0, rj.iz1, M))
            return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        const int kla = cd.LDA - 1 - cd.KU;
        op.dgbmv = static_cast<const double*>(rd.bands);
        op.dg_off = rd.offM;
        op.dg_lda = cd.LDA;
        op.dg_ku = cd.KU;
        op.dg_skip = st(dg)->dg_skip;
        KL += kla;
        KU += cd.KU;
        io.iz0 = rd.iz0;  // the chain reads b through the dgbmv's input window
        io.iz1 = rd.iz1;
    }
    if (bl) {
        const PfSolveConfiguration& cb = bl->configuration;
        Resolved rb;
        if ((res = resolve(bl, blp, rb)) != PFSOLVE_SUCCESS) return res;
        const int bt = cb.block % 10, sk = cb.block / 100;
        if ((int64_t)cb.size[0] != M || rb.bands != rj.rhs) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        if (!trivial_window(rj.oz0, rj.oz1, M) || !trivial_window(rb.iz0, rb.iz1, M))
            return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        if (sk == 1 && !(cb.jw_control_bitmask & RUNTIME_SCALEC) && cb.scaleC == 0.0)
            return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        if (bt == 1) {
            if (rb.offM != rj.offS || rb.iS != rj.oS || rb.batch != rj.batch) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
            LOUT = LAY_REAL;
        } else if (bt == 7) {
            // XXII pairs (real rows 2y, 2y+1 of the JW batch) -> packed complex y
            if (2 * rb.offM != rj.offS || rb.iS != rj.oS || 2 * rb.batch != rj.batch)
                return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
            LIN = LAY_XXII;
            LOUT = LAY_PACKED;
            io.in_off = rj.offS;
            io.nsys = rb.batch;
        } else {
            return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        }
        io.out = static_cast<double*>(rb.rhs);
        io.out_off = rb.offS;
        io.out_stride = rb.oS;
        io.oz0 = rb.oz0;
        io.oz1 = rb.oz1;
        io.accumulate = ((cb.block / 10) % 10) == 2;
        if (sk) {
            SCALE = 1;
            op.scale_kind = sk;
            op.lshift = cb.lshift;
            op.scale_s = rb.scaleC;
        }
    }
    // plan for the fused variant
    for (const AppState::ChainPlan& cp : sj->chain_plans) {
        if (cp.KL != KL || cp.KU != KU || cp.sv != L.sv || cp.LIN != LIN || cp.LOUT != LOUT || cp.SCALE != SCALE)
            continue;
        AppState t;
        t.num_sms = sj->num_sms;
        t.variant = cp.variant;
        t.R = cp.R;
        t.W = cp.W;
        t.G = cp.G;
        t.max_blocks = cp.max_blocks;
        t.stream_v = cp.stream_v;
        t.stream_G = cp.stream_G;
        t.stream_max_blocks = cp.stream_max_blocks;
        t.stream_nbuf = cp.stream_nbuf;
        return launch_jw_variant(&t, op, io, stream);
    }
    AppState t;
    t.num_sms = sj->num_sms;
    t.device = sj->device;
    t.prec = sj->prec;
    t.refine_sweeps = sj->refine_sweeps;
    t.KL = KL;
    t.KU = KU;
    t.sv = L.sv;
    t.R = pick_rows_per_thread(M, cj.rowsPerThread);
    if (t.R < 4) t.R = 4;
    t.R_fixed = cj.rowsPerThread != 0 && cj.rowsPerThread != 32;
    t.R_req = cj.rowsPerThread;
    t.no_stream = cj.kernelPath == 1;
    t.nbuf_req = cj.stagingBuffers;
    if (finish_variant(&t, M, LIN, LOUT, SCALE) != PFSOLVE_SUCCESS) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    sj->chain_plans.push_back(AppState::ChainPlan{KL, KU, L.sv, LIN, LOUT, SCALE, t.variant, t.R, t.W, t.G,
                                                  t.max_blocks, t.stream_v, t.stream_G, t.stream_max_blocks,
                                                  t.stream_nbuf});
    return launch_jw_variant(&t, op, io, stream);
}

}  // namespace

extern "C" PfSolveResult PfSolveAppendChain(PfSolveApplication** apps, PfSolveLaunchParams** lps, int n,
                                            int allowUnfused)
{
    if (!apps || n < 1) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    for (int i = 0; i < n; i++)
        if (!apps[i] || !apps[i]->internal) return PFSOLVE_ERROR_PLAN_NOT_INITIALIZED;
    PfSolveApplication *dg = nullptr, *jw = nullptr, *bl = nullptr;
    const PfSolveLaunchParams *dlp = nullptr, *jlp = nullptr, *blp = nullptr;
    bool pattern = true;
    int i = 0;
    if (i < n && st(apps[i])->kind == APP_DGBMV) { dg = apps[i]; dlp = lps ? lps[i] : nullptr; i++; }
    if (i < n && st(apps[i])->kind == APP_JW) { jw = apps[i]; jlp = lps ? lps[i] : nullptr; i++; }
    else pattern = false;
    if (i < n && st(apps[i])->kind == APP_BLOCK) { bl = apps[i]; blp = lps ? lps[i] : nullptr; i++; }
    if (i != n) pattern = false;
    PfSolveResult r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    const bool fusable = pattern && !st(jw)->alt && st(jw)->K == 1;  // ALT and K-step plans run alone
    if (fusable && (dg || bl)) {
        cudaStream_t stream = pick_stream(jw);
        r = append_chain_fused(dg, dlp, jw, jlp, bl, blp, stream);
        if (r == PFSOLVE_SUCCESS) record_stream_event(jw, stream);
    } else if (pattern && n == 1) {
        r = PfSolveAppend(jw, 0, lps ? lps[0] : nullptr);
    }
    if (r == PFSOLVE_ERROR_UNSUPPORTED_COMBINATION && allowUnfused) {
        for (int k = 0; k < n; k++) {
            r = PfSolveAppend(apps[k], 0, lps ? lps[k] : nullptr);
            if (r != PFSOLVE_SUCCESS) return r;
        }
    }
    return r;
}

// ---------------------------------------------------------------------------
// Uneven batches: many matrices of different sizes, one persistent launch.
#include <vector>

struct PfSolveBatch {
    PfSolveBatchDesc desc;
    int device = 0, num_sms = 0;
    int KL = 0, KU = 0, SV = 0, LIN = 0, LOUT = 0, SCALE = 0, PREC = 0;
    int64_t Mmax = 0;
    int R = 8, W = 1, G = 1, spi = 64;
    int max_blocks = 0;
    const BatchVariant* variant = nullptr;
    // sweep kernel (one system per lane) in use; nullptr: the group kernel
    const BatchSeqVariant* seq = nullptr;
    bool seq_ok = false;  // every entry allows the sweep kernel
    int seq_shape = 0;    // its compiled shape (rows per chunk, buffers, warps)
    // the sweep kernel's per-entry tensor maps and coefficient rows (written
    // by its pre-pass each launch)
    double* d_coefs = nullptr;
    BatchSeqEntry* d_seq = nullptr;
    std::vector<BatchEntryDev> entries;
    std::vector<WorkItem> items;
    BatchEntryDev* d_entries = nullptr;
    WorkItem* d_items = nullptr;
    size_t d_items_cap = 0;
    unsigned int* d_counter = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    double tuned_ms = 0.0;
};

namespace {

void batch_drop_graph(PfSolveBatch* b)
{
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
}

PfSolveResult batch_build_items(PfSolveBatch* b, int spi)
{
    b->items.clear();
    for (size_t e = 0; e < b->entries.size(); ++e) {
        const int64_t n = b->entries[e].io.nsys;
        for (int64_t y0 = 0; y0 < n; y0 += spi) {
            WorkItem w;
            w.entry = (int)e;
            w.pad = 0;
            w.y0 = y0;
            w.y1 = std::min<int64_t>(n, y0 + spi);
            b->items.push_back(w);
        }
    }
    // largest work first (bytes ~ rows x systems), ties by entry for locality
    std::stable_sort(b->items.begin(), b->items.end(), [&](const WorkItem& x, const WorkItem& y) {
        const int64_t cx = b->entries[x.entry].op.M * (x.y1 - x.y0);
        const int64_t cy = b->entries[y.entry].op.M * (y.y1 - y.y0);
        return cx > cy;
    });
    if (b->items.size() > b->d_items_cap) {
        if (b->d_items) cudaFree(b->d_items);
        b->d_items = nullptr;
        if (cudaMalloc(&b->d_items, b->items.size() * sizeof(WorkItem)) != cudaSuccess)
            return PFSOLVE_ERROR_FAILED_TO_ALLOCATE;
        b->d_items_cap = b->items.size();
    }
    if (!b->items.empty() &&
        cudaMemcpy(b->d_items, b->items.data(), b->items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice) !=
            cudaSuccess)
        return PFSOLVE_ERROR_FAILED_TO_COPY;
    b->spi = spi;
    return PFSOLVE_SUCCESS;
}

// The sweep kernel: FP64 bidiagonal (or matvec-only) steps whose V*A stays
// within rows i-1..i+1, XXII in, packed complex out, no accumulation; every
// entry's output 16-byte aligned and disjoint from its input (the sweep writes
// a chunk's results before it has read the later rows of the system).
bool batch_seq_allowed(const PfSolveBatch* b)
{
    if (b->PREC != PREC_F64 || b->KL > 1 || b->KU > 1 || b->SV == SV_TRI || b->LIN != LAY_XXII ||
        b->LOUT != LAY_PACKED)
        return false;
    for (const BatchEntryDev& e : b->entries) {
        if (e.io.accumulate) return false;
        const uintptr_t i0 = reinterpret_cast<uintptr_t>(e.io.in + e.io.in_off);
        const uintptr_t i1 = i0 + (uintptr_t)(2 * e.io.nsys * e.io.in_stride) * 8;
        const uintptr_t o0 = reinterpret_cast<uintptr_t>(e.io.out) + (uintptr_t)e.io.out_off * 16;
        const uintptr_t o1 = o0 + (uintptr_t)(e.io.nsys * e.io.out_stride) * 16;
        if ((o0 & 15) != 0 || e.io.out_stride < e.io.M || (e.io.nsys > 0 && i0 < o1 && o0 < i1)) return false;
    }
    return true;
}

PfSolveResult batch_configure_seq(PfSolveBatch* b, int shape)
{
    const BatchSeqVariant* v = find_batch_seq_variant(b->SV, shape);
    if (!v) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    if (!b->d_seq) {
        // per entry: tensor maps and its first coefficient row
        std::vector<BatchSeqEntry> sq(b->entries.size());
        int64_t rows = 0;
        for (size_t e = 0; e < b->entries.size(); ++e) {
            memset(&sq[e], 0, sizeof(BatchSeqEntry));
            const JwIO& io = b->entries[e].io;
            if (io.nsys > 0 && !encode_batch_seq_maps(io, &sq[e])) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
            sq[e].coef_off = rows;
            rows += batch_seq_rows(b->entries[e].op.M);
        }
        if (cudaMalloc(&b->d_coefs, std::max<int64_t>(rows, 1) * 48) != cudaSuccess ||
            cudaMalloc(&b->d_seq, std::max<size_t>(sq.size(), 1) * sizeof(BatchSeqEntry)) != cudaSuccess) {
            cudaGetLastError();
            return PFSOLVE_ERROR_FAILED_TO_ALLOCATE;
        }
        if (!sq.empty() &&
            cudaMemcpy(b->d_seq, sq.data(), sq.size() * sizeof(BatchSeqEntry), cudaMemcpyHostToDevice) != cudaSuccess)
            return PFSOLVE_ERROR_FAILED_TO_COPY;
    }
    const size_t smem = batch_seq_smem(v);
    if (!allow_max_smem(v->func)) return PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, v->func, 32 * v->NW, smem) != cudaSuccess ||
        blocks < 1) {
        cudaGetLastError();
        return PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE;
    }
    b->seq = v;
    b->seq_shape = shape;
    b->variant = nullptr;
    b->R = 0;
    b->W = 0;
    b->G = v->NW;
    b->max_blocks = blocks * b->num_sms;
    return PFSOLVE_SUCCESS;
}

PfSolveResult batch_configure(PfSolveBatch* b, int R)
{
    int64_t W = (b->Mmax + 32 * (int64_t)R - 1) / (32 * (int64_t)R);
    if (W < 1) W = 1;
    if (W > 8) return PFSOLVE_ERROR_UNSUPPORTED_FFT_LENGTH;
    const BatchVariant* v = find_batch_variant(R, b->KL, b->KU, b->SV, b->LIN, b->LOUT, b->SCALE, b->PREC);
    if (!v) return PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
    const int G = std::max(1, 8 / (int)W);
    const size_t smem = v->smem_bytes((int)W, G);
    if (smem > 48 * 1024 && !allow_max_smem(v->func)) return PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, v->func, 32 * (int)W * G, smem) != cudaSuccess ||
        blocks < 1)
        return PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE;
    b->variant = v;
    b->seq = nullptr;
    b->R = R;
    b->W = (int)W;
    b->G = G;
    b->max_blocks = blocks * b->num_sms;
    return PFSOLVE_SUCCESS;
}

PfSolveResult batch_launch(PfSolveBatch* b, cudaStream_t stream)
{
    const int nitems = (int)b->items.size();
    if (nitems == 0) return PFSOLVE_SUCCESS;
    if (cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned int), stream) != cudaSuccess)
        return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    const int64_t want = (nitems + b->G - 1) / b->G;
    const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(want, b->max_blocks));
    if (b->seq) {
        b->seq->coefs((int)b->entries.size(), stream, b->d_entries, b->d_seq, b->d_coefs);
        b->seq->launch(dim3((unsigned)grid), batch_seq_smem(b->seq), stream, b->d_entries, b->d_seq, b->d_coefs,
                       b->d_items, nitems, b->d_counter);
        g_launches.fetch_add(2, std::memory_order_relaxed);
        if (cudaPeekAtLastError() != cudaSuccess) {
            cudaGetLastError();
            return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
        }
        return PFSOLVE_SUCCESS;
    }
    const size_t smem = b->variant->smem_bytes(b->W, b->G);
    b->variant->launch(dim3((unsigned)grid), dim3(32 * b->W * b->G), smem, stream, b->d_entries, b->d_items, nitems,
                       b->d_counter, b->W);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();
        return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    }
    return PFSOLVE_SUCCESS;
}

}  // namespace

extern "C" {

PfSolveResult PfSolveBatchCreate(PfSolveBatch** out, CUdevice device, const PfSolveBatchDesc* desc,
                                 const PfSolveBatchEntry* entries, int nentries)
{
    if (!out || !desc || (nentries > 0 && !entries) || nentries < 0) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    *out = nullptr;
    PfSolveBatch* b = new (std::nothrow) PfSolveBatch();
    if (!b) return PFSOLVE_ERROR_MALLOC_FAILED;
    b->desc = *desc;
    b->device = device;
    auto fail = [&](PfSolveResult r) {
        PfSolveBatchDestroy(b);
        return r;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(PFSOLVE_ERROR_INVALID_DEVICE);
    if (cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return fail(PFSOLVE_ERROR_FAILED_TO_GET_ATTRIBUTE);
    if (desc->mixedPrecisionRefinement < 0 || desc->mixedPrecisionRefinement > 3)
        return fail(PFSOLVE_ERROR_INVALID_ARGUMENT);
    const int bt = desc->block % 10, sk = desc->block / 100;
    if (!(bt == 0 || bt == 1 || bt == 7) || ((desc->block / 10) % 10 != 0 && (desc->block / 10) % 10 != 2) || sk > 4)
        return fail(PFSOLVE_ERROR_UNSUPPORTED_COMBINATION);
    if (bt == 0 && desc->block != 0) return fail(PFSOLVE_ERROR_UNSUPPORTED_COMBINATION);
    PfSolveConfiguration c;
    memset(&c, 0, sizeof(c));
    c.upperBanded = desc->upperBanded;
    c.jw_type = desc->jw_type;
    c.M_size = 16;
    JwLayout L0;
    if (desc->jw_type < 10 || !jw_layout(c, false, false, 0, 0, L0)) return fail(PFSOLVE_ERROR_UNSUPPORTED_COMBINATION);
    b->SV = L0.sv;
    b->KL = (L0.mvj == MVJ_LOWER) ? 1 : 0;
    b->KU = (L0.mvj == MVJ_UPPER) ? 1 : 0;
    if (desc->LDA > 0) {
        if (desc->KU < 0 || desc->KU >= desc->LDA) return fail(PFSOLVE_ERROR_INVALID_ARGUMENT);
        b->KL += desc->LDA - 1 - desc->KU;
        b->KU += desc->KU;
    }
    b->LIN = (bt == 7) ? LAY_XXII : LAY_REAL;
    b->LOUT = (bt == 7) ? LAY_PACKED : LAY_REAL;
    b->SCALE = sk ? 1 : 0;
    b->PREC = (desc->mixedPrecisionRefinement > 0 && b->SV != SV_NONE) ? 1 : 0;
    for (int e = 0; e < nentries; ++e) {
        const PfSolveBatchEntry& en = entries[e];
        if (en.M < 1 || en.M > kMaxRows || en.nsys < 0 || !en.bands || !en.input || !en.output)
            return fail(PFSOLVE_ERROR_INVALID_ARGUMENT);
        if (desc->LDA > 0 && !en.dgbmvBands) return fail(PFSOLVE_ERROR_INVALID_ARGUMENT);
        c.M_size = en.M;
        JwLayout L;
        jw_layout(c, false, false, 0, 0, L);
        BatchEntryDev d;
        memset(&d, 0, sizeof(d));
        AppState tmp;
        tmp.refine_sweeps = 1 + desc->mixedPrecisionRefinement;
        fill_operator_common(&tmp, c, d.op);
        d.op.bands = static_cast<const double*>(en.bands);
        d.op.off_md = L.off_md;
        d.op.off_mo = L.off_mo;
        d.op.off_sl = L.off_sl;
        d.op.off_su = L.off_su;
        d.op.mvj = L.mvj;
        d.op.scaleC = en.scaleC;
        if (desc->LDA > 0) {
            d.op.dgbmv = static_cast<const double*>(en.dgbmvBands);
            d.op.dg_off = 0;
            d.op.dg_lda = desc->LDA;
            d.op.dg_ku = desc->KU;
        }
        d.op.scale_kind = sk;
        d.op.lshift = en.lshift;
        d.op.scale_s = en.scaleS;
        d.io.in = static_cast<const double*>(en.input);
        d.io.out = static_cast<double*>(en.output);
        d.io.in_stride = en.inputStride;
        d.io.out_stride = en.outputStride;
        d.io.iz0 = 0;
        d.io.iz1 = INT64_MAX / 4;
        d.io.oz0 = 0;
        d.io.oz1 = INT64_MAX / 4;
        d.io.nsys = en.nsys;
        d.io.M = en.M;
        d.io.accumulate = ((desc->block / 10) % 10) == 2;
        b->entries.push_back(d);
        b->Mmax = std::max<int64_t>(b->Mmax, en.M);
    }
    if (cudaMalloc(&b->d_counter, sizeof(unsigned int)) != cudaSuccess) return fail(PFSOLVE_ERROR_FAILED_TO_ALLOCATE);
    if (!b->entries.empty()) {
        if (cudaMalloc(&b->d_entries, b->entries.size() * sizeof(BatchEntryDev)) != cudaSuccess)
            return fail(PFSOLVE_ERROR_FAILED_TO_ALLOCATE);
        if (cudaMemcpy(b->d_entries, b->entries.data(), b->entries.size() * sizeof(BatchEntryDev),
                       cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(PFSOLVE_ERROR_FAILED_TO_COPY);
    }
    b->seq_ok = batch_seq_allowed(b);
    if (desc->sweepRows) {
        // the sweep kernel with the first compiled shape of that chunk depth
        PfSolveResult r = PFSOLVE_ERROR_UNSUPPORTED_COMBINATION;
        for (int shape = 0; b->seq_ok && shape < kBatchSeqShapes && r != PFSOLVE_SUCCESS; ++shape) {
            const BatchSeqVariant* v = find_batch_seq_variant(b->SV, shape);
            if (v && v->CH == desc->sweepRows) r = batch_configure_seq(b, shape);
        }
        if (r == PFSOLVE_SUCCESS) r = batch_build_items(b, 32);
        if (r != PFSOLVE_SUCCESS) return fail(r);
        *out = b;
        return PFSOLVE_SUCCESS;
    }
    // default shape: the sweep kernel where the batch allows it (items of one
    // warp's 32 systems), else the group kernel with 8 (or 4) rows per thread
    if (b->seq_ok && !desc->rowsPerThread && desc->systemsPerItem <= 0 &&
        batch_configure_seq(b, 0) == PFSOLVE_SUCCESS) {
        PfSolveResult r = batch_build_items(b, 32);
        if (r != PFSOLVE_SUCCESS) return fail(r);
        *out = b;
        return PFSOLVE_SUCCESS;
    }
    int R = desc->rowsPerThread ? desc->rowsPerThread : 8;
    PfSolveResult r = batch_configure(b, R);
    if (r != PFSOLVE_SUCCESS && !desc->rowsPerThread) r = batch_configure(b, 4);
    if (r != PFSOLVE_SUCCESS) return fail(r);
    int spi = desc->systemsPerItem;
    if (spi <= 0) {
        // about 4 items per resident group keeps the queue balanced
        int64_t total = 0;
        for (const auto& e : b->entries) total += e.io.nsys;
        const int64_t groups = std::max<int64_t>(1, (int64_t)b->max_blocks * b->G);
        spi = (int)std::max<int64_t>(8, std::min<int64_t>(256, total / (4 * groups) + 1));
    }
    if ((r = batch_build_items(b, spi)) != PFSOLVE_SUCCESS) return fail(r);
    *out = b;
    return PFSOLVE_SUCCESS;
}

PfSolveResult PfSolveBatchAppend(PfSolveBatch* b, cudaStream_t stream)
{
    if (!b) return PFSOLVE_ERROR_PLAN_NOT_INITIALIZED;
    if (b->graph_exec) {
        if (cudaGraphLaunch(b->graph_exec, stream) != cudaSuccess) return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
        g_launches.fetch_add(b->seq ? 2 : 1, std::memory_order_relaxed);  // kernels in the graph
        return PFSOLVE_SUCCESS;
    }
    return batch_launch(b, stream);
}

PfSolveResult PfSolveBatchCaptureGraph(PfSolveBatch* b, cudaStream_t stream)
{
    if (!b) return PFSOLVE_ERROR_PLAN_NOT_INITIALIZED;
    if (!stream) return PFSOLVE_ERROR_INVALID_ARGUMENT;  // the legacy default stream cannot be captured
    batch_drop_graph(b);
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    const uint64_t before = g_launches.load();
    PfSolveResult r = batch_launch(b, stream);
    g_launches.store(before);  // capturing enqueues nothing
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(stream, &graph);
    if (r != PFSOLVE_SUCCESS || ce != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        return r != PFSOLVE_SUCCESS ? r : PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    }
    if (cudaGraphInstantiate(&b->graph_exec, graph, 0) != cudaSuccess) {
        cudaGraphDestroy(graph);
        b->graph_exec = nullptr;
        return PFSOLVE_ERROR_FAILED_TO_LAUNCH_KERNEL;
    }
    b->graph = graph;
    return PFSOLVE_SUCCESS;
}

PfSolveResult PfSolveBatchAutotune(PfSolveBatch* b, cudaStream_t stream, int iterations)
{
    if (!b) return PFSOLVE_ERROR_PLAN_NOT_INITIALIZED;
    for (const auto& e : b->entries)
        if ((const void*)e.io.in == (const void*)e.io.out) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    if (iterations < 1) iterations = 3;
    batch_drop_graph(b);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int bestR = b->R, bestSpi = b->spi, bestShape = b->seq_shape;
    auto time_shape = [&]() -> double {
        if (batch_launch(b, stream) != PFSOLVE_SUCCESS) return 1e300;  // warm-up
        cudaEventRecord(e0, stream);
        for (int it = 0; it < iterations; ++it) batch_launch(b, stream);
        cudaEventRecord(e1, stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) return 1e300;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms / iterations;
    };
    // the sweep kernel (rows per thread reported as 0), one warp's 32 systems per item
    for (int shape = 0; shape < kBatchSeqShapes; ++shape) {
        if (!b->seq_ok || batch_configure_seq(b, shape) != PFSOLVE_SUCCESS) continue;
        if (batch_build_items(b, 32) != PFSOLVE_SUCCESS) continue;
        const double per = time_shape();
        if (per < best) {
            best = per;
            bestR = 0;
            bestSpi = 32;
            bestShape = shape;
        }
    }
    for (int R : {4, 8, 16, 2}) {
        if (batch_configure(b, R) != PFSOLVE_SUCCESS) continue;
        for (int spi : {16, 32, 64, 128}) {
            if (batch_build_items(b, spi) != PFSOLVE_SUCCESS) continue;
            const double per = time_shape();
            if (per < best) {
                best = per;
                bestR = R;
                bestSpi = spi;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PfSolveResult r = bestR ? batch_configure(b, bestR) : batch_configure_seq(b, bestShape);
    if (r == PFSOLVE_SUCCESS) r = batch_build_items(b, bestSpi);
    if (r == PFSOLVE_SUCCESS) b->tuned_ms = best;
    return r;
}

PfSolveResult PfSolveBatchGetSweepShape(const PfSolveBatch* b, int* rowsPerChunk, int* buffers, int* warpsPerCTA)
{
    if (!b) return PFSOLVE_ERROR_PLAN_NOT_INITIALIZED;
    if (rowsPerChunk) *rowsPerChunk = b->seq ? b->seq->CH : 0;
    if (buffers) *buffers = b->seq ? b->seq->NBUF : 0;
    if (warpsPerCTA) *warpsPerCTA = b->seq ? b->seq->NW : 0;
    return PFSOLVE_SUCCESS;
}

PfSolveResult PfSolveBatchGetShape(const PfSolveBatch* b, int* R, int* W, int* spi, int* items, double* ms)
{
    if (!b) return PFSOLVE_ERROR_PLAN_NOT_INITIALIZED;
    if (R) *R = b->R;
    if (W) *W = b->W;
    if (spi) *spi = b->spi;
    if (items) *items = (int)b->items.size();
    if (ms) *ms = b->tuned_ms;
    return PFSOLVE_SUCCESS;
}

void PfSolveBatchDestroy(PfSolveBatch* b)
{
    if (!b) return;
    batch_drop_graph(b);
    if (b->d_entries) cudaFree(b->d_entries);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_counter) cudaFree(b->d_counter);
    if (b->d_coefs) cudaFree(b->d_coefs);
    if (b->d_seq) cudaFree(b->d_seq);
    delete b;
}

}  // extern "C"
