/*
 * jw_oracle.h -- CPU restatement of PfSolve's Jones-Worland (JW) step, its dgbmv
 * band matvec and its block/Scale kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark call it.  The product
 * (libpfsolve_b200.so) never links, loads or calls it.
 *
 * Every routine restates the reference's algorithm in plain C from the generator
 * sources cited beside it (paths relative to the PfSolve project root).  The
 * arithmetic runs in __float128 (the "q" entry points: the accuracy oracle that
 * stands in for the reference's 128-bit mpir verification,
 * benchmark_scripts/vkFFT_scripts/src/sample_0_benchmark_VkFFT_single.cpp:353-435)
 * and in double (the "d" entry points: the reference's own CPU verification path,
 * a sequential Thomas/back-substitution per right-hand side,
 * sample_0_benchmark_VkFFT_single.cpp:437-460 and
 * sample_1_benchmark_VkFFT_double_JW.cpp:243-259).
 */
#ifndef PFSOLVE_JW_ORACLE_H
#define PFSOLVE_JW_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Bitfield values of PfSolveConfiguration.jw_control_bitmask
 * (PfSolve/pfSolve_Structs/pfSolve_Structs.h:73-81). */
#define PFO_RUNTIME_OFFSETM 2
#define PFO_RUNTIME_OFFSETV 4
#define PFO_RUNTIME_OFFSETSOLUTION 8
#define PFO_RUNTIME_INPUTZEROPAD 16
#define PFO_RUNTIME_OUTPUTZEROPAD 32
#define PFO_RUNTIME_SCALEC 64
#define PFO_RUNTIME_INPUTBUFFERSTRIDE 128
#define PFO_RUNTIME_OUTPUTBUFFERSTRIDE 256

/* Plan-time values (PfSolveConfiguration) and launch-time values
 * (PfSolveLaunchParams) exactly as a caller would set them; the oracle resolves
 * which one applies from `bitmask`, the way the plan does
 * (PfSolve/pfSolve_PlanManagement/pfSolve_Plans/pfSolve_Plan_JonesWorland.h:387-526). */
typedef struct {
    int64_t M;                 /* M_size: rows per system */
    int64_t batch;             /* number of right-hand sides (size[1]*size[2]) */
    int32_t upperBanded;       /* 0, 1 or 2 */
    int32_t jw_type;           /* 10..13 (jw_type % 10 selects matvec/solve) */
    int64_t bitmask;           /* jw_control_bitmask */
    /* plan-time values */
    int64_t cfg_offsetM, cfg_offsetV, cfg_offsetSolution;
    int64_t cfg_inputZeropad[2], cfg_outputZeropad[2];
    int64_t cfg_inputBufferStride, cfg_outputBufferStride;
    double cfg_scaleC;
    /* launch-time values */
    int64_t run_offsetM, run_offsetV, run_offsetSolution;
    int64_t run_inputZeropad[2], run_outputZeropad[2];
    int64_t run_inputBufferStride, run_outputBufferStride;
    double run_scaleC;
    /* 1: bands are stored in the reference's register-major order (reorder_i0) */
    int32_t bandsPermuted;
    /* dgbmv: LDA bands (band-major), KU super-, KL sub-diagonals */
    int32_t LDA, KU, KL;
    /* block kernel */
    int32_t block, lshift;
    int64_t size0, size1;      /* block kernel extents */
    int32_t ALT_dgbmv;         /* dgbmv: drop alternate bands (stride-2 couplings) */
} pfo_params;

/* Operator kinds of one JW step after the band offsets are resolved. */
enum { PFO_MV_NONE = 0, PFO_MV_DIAG = 1, PFO_MV_UPPER = 2, PFO_MV_LOWER = 3 };
enum { PFO_SV_NONE = 0, PFO_SV_LOWER = 1, PFO_SV_UPPER = 2, PFO_SV_TRI = 3 };

/* Storage position of logical row i for the register-major band layout.
 * Restates reorder_i0 (pfSolve_Plan_JonesWorland.h:66-142) for the CUDA
 * backend (warp 32, Msplit 256 for M > 4352). */
int64_t pfo_reorder_i0(int64_t i, int64_t M, int64_t Msplit0);

/* Resolve the band offsets and operator kinds of one JW step (K = 1) and return
 * natural-order copies of the bands it uses (each array has M entries; unused
 * arrays are left untouched).  Returns 0, or -1 for a combination the reference
 * does not define (upperBanded 2 with jw_type%10 in {0,1}).
 * Follows pfSolve_KernelsLevel2/pfSolve_JonesWorland.h:117-353. */
int pfo_jw_operator(const pfo_params* p, const double* bands, int* mv_kind, int* sv_kind,
                    double* mv_d, double* mv_o, double* sv_l, double* sv_u);

/* One JW step over all right-hand sides, in place on `rhs` (FP64 storage, as
 * the FP64 kernel sees it).  q: __float128 arithmetic; d: double arithmetic.
 * nthreads > 1 splits right-hand sides over OpenMP threads.  Returns 0 or -1. */
int pfo_jw_step_q(const pfo_params* p, const double* bands, double* rhs, int nthreads);
int pfo_jw_step_d(const pfo_params* p, const double* bands, double* rhs, int nthreads);
/* Same step for FP32 storage (bands and rhs float), computed in __float128. */
int pfo_jw_step_q_f32(const pfo_params* p, const float* bands, float* rhs, int nthreads);
/* Double-double storage: every value is a pair {hi, lo} (the reference's
 * pf_quad2, pfSolve_KernelsLevel0/pfSolve_KernelUtils.h:122-150).  Computed in
 * __float128 and rounded back to {hi, lo}. */
int pfo_jw_step_q_dd(const pfo_params* p, const double* bands_dd, double* rhs_dd, int nthreads);

/* ALT stride-2 mode (jw_type / 100 % 10 == 1), K = 1, FP64: the even and the
 * odd rows form two independent systems with neighbours r -+ 2; bands in the
 * ALT register layout (pfo_alt_position), R T entries apart.  Returns -1 for
 * launch-time band offsets (the reference rescales only plan-time ones). */
int64_t pfo_alt_position(int64_t r, int64_t M);
int pfo_jw_step_alt_q(const pfo_params* p, const double* bands, double* rhs, int nthreads);

/* K consecutive JW steps (numConsecutiveJWIterations = K, 2 <= K <= 8) on
 * real FP64 systems, in __float128 ("q") or double ("d").  `bands` holds
 * `nbuf` buffer pointers: one per step (nbuf >= K, the reference's
 * useMultipleInputBuffers) or a single buffer read by every step (nbuf = 1).
 * Returns 0, or -1 for a combination the reference leaves undefined.
 * Follows pfSolve_KernelsLevel2/pfSolve_JonesWorland.h:108-374. */
#define PFO_MAX_STEPS 8
typedef struct {
    int64_t M, r;              /* rows of the step; register count of the band order */
    int32_t mv, sv, diag;      /* operator kinds; whether the matvec diagonal is applied */
    int64_t off_md, off_mo, off_sl, off_su;
} pfo_step;
int64_t pfo_steps_registers(int64_t M, int upperBanded, int K);
int pfo_jw_steps_layout(const pfo_params* p, int K, int s, pfo_step* st);
int pfo_jw_steps_q(const pfo_params* p, int K, int nbuf, const double* const* bands, double* rhs, int nthreads);
int pfo_jw_steps_d(const pfo_params* p, int K, int nbuf, const double* const* bands, double* rhs, int nthreads);

/* General banded matvec y = A x, in place on rhs, A in band-major storage
 * A[offsetM + j*M + c] (pfSolve_KernelsLevel1/pfSolve_MatVecMul.h:383-446,
 * pfSolve_KernelsLevel2/pfSolve_dgbmv.h:38-112). */
/* 1 when ALT_dgbmv drops band j of a dgbmv application. */
int pfo_dgbmv_band_dropped(const pfo_params* p, int64_t j);
int pfo_dgbmv_q(const pfo_params* p, const double* A, double* rhs, int nthreads);
int pfo_dgbmv_d(const pfo_params* p, const double* A, double* rhs, int nthreads);

/* Block copy/convert/scale kernel (pfSolve_KernelsLevel2/pfSolve_block.h:37-115,
 * pfSolve_KernelsLevel1/pfSolve_ReadWrite.h:2275-2371,
 * pfSolve_KernelsLevel1/pfSolve_RegistersScaleC.h:27-201), FP64 storage,
 * out of place from `in` to `out`.  Returns 0 or -1 (undefined combination). */
int pfo_block_q(const pfo_params* p, const double* in, double* out);

/* The per-row factor of Scale{C,D,SphLaplA,SphLaplB} for row x (block/100 in
 * 1..4), runtime-scaleC form (pfSolve_RegistersScaleC.h:27-201). */
double pfo_scale_factor(int kind, int64_t x, int lshift, double s);

/* Relative errors of `a` against `ref` over the rows [0, M) of every system:
 * max over systems of ||a-ref||_2/||ref||_2, and max|a-ref| / max|ref|. */
void pfo_rel_errors(const double* a, const double* ref, int64_t M, int64_t batch, int64_t stride,
                    int64_t offset, double* rel_l2_max, double* rel_max);

/* Same for double-double storage: every value a {hi, lo} pair. */
void pfo_rel_errors_dd(const double* a, const double* ref, int64_t M, int64_t batch, int64_t stride,
                       int64_t offset, double* rel_l2_max, double* rel_max);

/* The radial DCT step that feeds the JW chain, batched over rows of N points:
 * type 2 (REDFT10) or 3 (REDFT01) in FFTW's unnormalized definitions,
 *   type 2: X_k = 2 sum_{n=0}^{N-1} x_n cos(pi k (2n+1) / (2N)),
 *   type 3: X_k = x_0 + 2 sum_{n=1}^{N-1} x_n cos(pi n (2k+1) / (2N)),
 * so that type 3 applied to type 2 is 2N times the identity.  PfSolve carries
 * the selector (PfSolveConfiguration.performDCT, pfSolve_Structs.h:272) from the
 * VkFFT it grew out of; the transform itself is VkFFT's, which follows FFTW's
 * definitions.  Direct O(N^2) sums in __float128, the angles reduced exactly
 * modulo 4N.  Row y is read at in + y*in_stride and written at out +
 * y*out_stride (out of place).  Returns 0, or -1 for a type other than 2, 3. */
int pfo_dct_q(int type, int64_t N, int64_t nsys, const double* in, int64_t in_stride, double* out,
              int64_t out_stride, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
