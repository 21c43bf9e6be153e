// jw_types.h -- host/device descriptors of one fused JW step launch.
#pragma once
#include <cstdint>

namespace pfb {

enum : int { SV_NONE = 0, SV_LOWER = 1, SV_UPPER = 2, SV_TRI = 3 };
enum : int { LAY_REAL = 0, LAY_XXII = 1, LAY_PACKED = 2 };
enum : int { MVJ_NONE = 0, MVJ_DIAG = 1, MVJ_UPPER = 2, MVJ_LOWER = 3 };
// Arithmetic of a kernel variant: FP64; FP32 solve + FP64 refinement;
// double-double on double-double storage; double-double on FP64 storage;
// FP32 on FP32 storage (the reference's default precision); FP64 on FP32
// storage (its doublePrecisionFloatMemory).
enum : int { PREC_F64 = 0, PREC_MIXED = 1, PREC_DD = 2, PREC_DD_F64MEM = 3, PREC_F32 = 4, PREC_F64_F32MEM = 5 };

// Precisions whose buffers (bands, dgbmv matrix, right-hand sides) hold FP32 values.
constexpr bool prec_f32_storage(int prec) { return prec == PREC_F32 || prec == PREC_F64_F32MEM; }

// The matrix side of a JW step: where the bands live and how to read them.
struct JwOperator {
    const double* bands;  // JW band buffer (FP64, or FP32 values when bands32)
    int64_t off_md, off_mo, off_sl, off_su;  // band offsets in elements (resolved on the host)
    int mvj;                                 // JW matvec kind (MVJ_*)
    int perm;                                // 1: bands in the reference's register-major order
    // reference band order (reorder_i0): rows per lane r, and for the pieces
    // of perm_piece rows (0: one piece) the count of lanes with ceil rows (m)
    // and the ceil / floor row counts; the partial last piece has its own
    int64_t perm_r, perm_m, perm_ceil, perm_floor;
    int64_t perm_piece, perm_lm, perm_lceil, perm_lfloor;
    const double* dgbmv;  // fused general band matrix (band-major), or nullptr
    int64_t dg_off;
    int dg_lda, dg_ku;
    uint64_t dg_skip;  // ALT_dgbmv: bit j set drops band j of the general band matrix
    int scale_kind, lshift;  // fused block Scale operator (0: none)
    double scale_s;
    double scaleC;  // multiplies solution row 0 when a solve runs
    int64_t M;
    int refine_sweeps;  // mixed precision: FP32 solves in total (1 + refinements)
    // ALT stride-2 mode: the rows of parity alt_h form the system (M counts
    // the full rows); bands in the ALT register layout of alt_T lanes x alt_R
    // rows (entry of row r = 2 e + h at (e % alt_R) alt_T + h alt_T/2 + e / alt_R)
    int alt, alt_h;
    int64_t alt_T, alt_R;
    int bands32;  // bands and the dgbmv matrix hold FP32 values (FP32-storage precisions)
};

// The DCT step (dct.cuh): rows of N points, in and out (possibly the same).
struct DctIO {
    const double* in;
    double* out;
    int64_t in_off, in_stride;    // elements
    int64_t out_off, out_stride;  // elements
    int64_t nsys;
};

// Streaming kernel: at most this many TMA staging buffers per group.
constexpr int kStMaxBuffers = 4;

// The data side: systems, layouts, keep-windows.
struct JwIO {
    const double* in;             // FP64 values, or FP32 values for the FP32-storage precisions
    double* out;
    int64_t in_off, in_stride;    // elements of the storage type (see LAY_*)
    int64_t out_off, out_stride;  // elements of the output type (real or complex, of the storage type)
    int64_t iz0, iz1;             // rows read as data: [iz0, iz1); others read as 0
    int64_t oz0, oz1;             // rows written: [oz0, oz1)
    int64_t nsys;                 // systems (real, or complex pairs)
    int64_t M;
    int accumulate;               // output += result
    int alt;                      // ALT mode: system 2y + h is the parity-h rows of row set y
    int plain;                    // long-system single pass: rows not 16-byte aligned, moved by plain loads/stores
    int nbuf;                     // streaming kernel: staging buffers per group (2..4; 0: 2)
};

// K consecutive steps in one kernel (numConsecutiveJWIterations = K).
constexpr int kMaxSteps = 8;

// One step, resolved on the host: its rows, band buffer and offsets, and the
// register-major band order of its rows (reorder_i0 for M_s rows with the
// plan's rows per lane, pfSolve_Plan_JonesWorland.h:66-142, 276-283, 342-346).
struct JwStepDesc {
    const double* bands;
    int64_t M;
    int64_t off_md, off_mo, off_sl, off_su;
    int diag;  // the matvec multiplies by the band diagonal (else by 1)
    int pad;
    int64_t perm_r, perm_m, perm_ceil, perm_floor;
};

struct JwSteps {
    int K;
    int perm;        // bands in the reference's register-major order
    double scaleC;   // solution row 0 after every solve
    int64_t M_in;    // rows read (M_0)
    int64_t M_out;   // rows written (M_{K-1})
    JwStepDesc st[kMaxSteps];
};

// Uneven batches: one descriptor per entry (systems sharing one matrix) and
// a work list of (entry, system range) items consumed through a counter.
struct BatchEntryDev {
    JwOperator op;
    JwIO io;
};
struct WorkItem {
    int entry;
    int pad;
    int64_t y0, y1;  // systems [y0, y1) of the entry
};

}  // namespace pfb
