// plan.h -- host-side planning helpers shared by the application API and the
// serving engine: band order, JW operator resolution, launch shapes.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <set>
#include <utility>

#include "../../include/pfsolve_b200.h"
#include "jw_variants.h"

namespace pfb {

// Let `func` use the device's full opt-in shared memory per block.  Set once
// per device and never lowered, so plans that launch one kernel with
// different shared-memory sizes do not undo each other's setting.
inline bool allow_max_smem(const void* func)
{
    static std::mutex mu;
    static std::set<std::pair<int, const void*>> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({dev, func})) return true;
    int maxopt = 0;
    if (cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, maxopt) != cudaSuccess)
        return false;
    done.insert({dev, func});
    return true;
}

// Count one kernel launch in PfSolveLaunchCount (and in
// PfSolveStreamingLaunchCount when it ran on the streaming kernel).
void note_launch(bool streaming);

// The reference's register-major band order (reorder_i0 with the CUDA
// backend's defaults, pfSolve_Plan_JonesWorland.h:66-142): systems of up to
// 4352 rows are one piece; longer ones are split into pieces of Msplit = 256
// rows, each permuted on its own (the last, partial piece with its own counts).
inline void set_band_order(int64_t M, JwOperator& op)
{
    const int64_t piece = (M > 4352) ? 256 : 0;
    const int64_t size1 = piece ? piece : M;
    int64_t warp = 64 * ((size1 + 1023) / 1024);
    if (size1 < 512) warp = 32;
    if (warp < 32) warp = 32;
    if (warp % 32) warp = 32 * ((warp + 31) / 32);
    int64_t r = (size1 + warp - 1) / warp;
    if (r < 1) r = 1;
    op.perm = 1;
    op.perm_r = r;
    op.perm_piece = piece;
    const int64_t full = piece ? piece : M;
    op.perm_m = full % r;
    op.perm_ceil = (full + r - 1) / r;
    op.perm_floor = full / r;
    const int64_t last = piece ? (M % piece) : 0;
    op.perm_lm = last % r;
    op.perm_lceil = (last + r - 1) / r;
    op.perm_lfloor = last / r;
}

// JW operator kinds for K = 1 (pfSolve_JonesWorland.h:117-353): which matvec,
// which solve, and where the bands sit.  Returns false for combinations the
// reference leaves undefined (upperBanded 2 with jw_type % 10 in {0, 1}).
struct JwLayout {
    int mvj, sv;
    int64_t off_md, off_mo, off_sl, off_su;
};

inline bool jw_layout(const PfSolveConfiguration& c, bool rtM, bool rtV, int64_t oM, int64_t oV, JwLayout& L)
{
    const int64_t M = c.M_size;
    const int jwt = c.jw_type % 10;
    L = JwLayout{MVJ_NONE, SV_NONE, 0, 0, 0, 0};
    if (c.upperBanded == 2) {
        // Only jw_type%10 == 3 is defined: with %10 == 2 the reference loads
        // the bands only for the matvec (:228-235, :269) and its solve is the identity.
        L.off_md = M; L.off_sl = 0; L.off_su = 2 * M;
        if (jwt == 3) { L.mvj = MVJ_DIAG; L.sv = SV_TRI; return true; }
        return false;
    }
    if (jwt == 2) L.mvj = MVJ_NONE;
    else if (jwt == 3) {
        // Offsets chosen with upperBanded flipped (:133-136, :203-206); the
        // solve reuses the off-diagonal band loaded with the matvec (no reload
        // when performTriSolve == 2, :337-344).
        L.mvj = MVJ_DIAG;
        if (c.upperBanded == 1) {
            L.off_md = rtM ? oM : M;
            L.sv = SV_LOWER;
            L.off_sl = rtM ? oM + M : 0;
        } else {
            L.off_md = rtM ? oM + M : 0;
            L.sv = SV_UPPER;
            L.off_su = rtM ? oM : M;
        }
        return true;
    } else if (c.upperBanded == 1) {
        L.mvj = MVJ_UPPER;
        L.off_md = rtM ? oM + M : 0;
        L.off_mo = rtM ? oM : M;
    } else {
        L.mvj = MVJ_LOWER;
        L.off_md = rtM ? oM : M;
        L.off_mo = rtM ? oM + M : 0;
    }
    if (jwt == 1) L.sv = SV_NONE;
    else if (c.upperBanded == 1) { L.sv = SV_LOWER; L.off_sl = rtV ? oV : 2 * M; }
    else { L.sv = SV_UPPER; L.off_su = rtV ? oV : 2 * M; }
    return true;
}

// Groups per CTA for variant v at W warps per system: the count that keeps the
// most groups resident per SM (shared memory, registers and the variant's
// launch bound permitting).  Returns false when nothing fits.
inline bool choose_groups(const JwVariant* v, int W, int num_sms, int& G_out, int& max_blocks)
{
    int best = 0, bestG = 0, bestBlocks = 0;
    for (int G = 1; 32 * W * G <= v->max_threads; ++G) {
        const size_t smem = v->smem_bytes(W, G);
        if (smem > 227 * 1024) break;
        if (smem > 48 * 1024 && !allow_max_smem(v->func)) break;
        int blocks = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, v->func, 32 * W * G, smem) != cudaSuccess)
            break;
        if (blocks * G > best) {
            best = blocks * G;
            bestG = G;
            bestBlocks = blocks;
        }
    }
    if (best == 0) return false;
    G_out = bestG;
    max_blocks = bestBlocks * num_sms;
    return true;
}

}  // namespace pfb
