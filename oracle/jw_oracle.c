/*
 * jw_oracle.c -- CPU restatement of PfSolve's Jones-Worland step (see jw_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for parity tests, smoke() and the CPU
 * baseline of bench.py.  Not part of the product; nothing in libpfsolve_b200.so
 * links or calls it.
 *
 * File references are relative to the PfSolve project root.
 */
#include "jw_oracle.h"

#include <math.h>
#include <quadmath.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef __float128 q_t;

/* ------------------------------------------------------------------------- */
/* Register-major band layout.
 * reorder_i0 (pfSolve_Plan_JonesWorland.h:66-142): the kernel gives each lane
 * r = ceil(M / T) consecutive rows (T = 32 below 512 rows, else 64*ceil(M/1024);
 * pfSolve_Plan_JonesWorland.h:311-346) and loads band register j of every lane
 * with one coalesced access, so row t*r + j is stored at S_j + t where S_j
 * counts the rows held by registers 0..j-1 (ceil(M/r) lanes for j < M%r, else
 * floor(M/r)).  Systems longer than 4352 rows are split into Msplit0-row
 * pieces, each permuted on its own. */
int64_t pfo_reorder_i0(int64_t i, int64_t M, int64_t Msplit0)
{
    if (Msplit0 == 0) Msplit0 = 256;
    int64_t size0 = M, size1 = M;
    if (M > 4352) { size0 = Msplit0; size1 = Msplit0; }
    int64_t warp = 64 * ((size1 + 1023) / 1024);
    if (size1 < 512) warp = 32;
    if (warp < 32) warp = 32;
    if (warp % 32) warp = 32 * ((warp + 31) / 32);
    int64_t r = (size1 + warp - 1) / warp;
    int64_t piece = (i / size0) * size0;
    int64_t li = i % size0;
    if (((i / size0) + 1) * size0 > M) size0 = M % size0;
    int64_t t = li / r, j = li % r;
    int64_t m = size0 % r, ceil_n = (size0 + r - 1) / r, floor_n = size0 / r;
    int64_t pos = t;
    if (j < m) pos += j * ceil_n;
    else pos += m * ceil_n + (j - m) * floor_n;
    return pos + piece;
}

/* ------------------------------------------------------------------------- */
/* Resolution of plan-time vs launch-time values (pfSolve_Plan_JonesWorland.h:387-526). */
static int64_t rv(const pfo_params* p, int64_t bit, int64_t cfg, int64_t run)
{
    return (p->bitmask & bit) ? run : cfg;
}

/* Keep-window test of PfConfigureZeropad (pfSolve_KernelsLevel0/pfSolve_Zeropad.h:306-377):
 * launch-time windows keep [z0, z1); plan-time windows treat 0 as "no bound". */
static int keep(int64_t i, int64_t z0, int64_t z1, int runtime)
{
    if (runtime) return (i >= z0) && (i < z1);
    if (z0) return (i >= z0) && ((z1 == 0) || (i < z1));
    if (z1) return i < z1;
    return 1;
}

typedef struct {
    int mv, sv;
    int64_t off_md, off_mo, off_sl, off_su; /* band offsets (elements) */
} jw_layout;

/* Band offsets for K = 1 (pfSolve_JonesWorland.h:117-207 for the matvec
 * operand, :269-353 for the solve operand).  Plan-time offsetM/offsetV are
 * not added by the reference (the additions are commented out at :161-162,
 * :191-192, :291-295, :321-324); only the RUNTIME_OFFSETM/V forms move the
 * bands, and with the runtime forms the two matvec bands swap places
 * (:156-157 and :186-187). */
static int jw_resolve(const pfo_params* p, jw_layout* L)
{
    const int64_t M = p->M;
    const int jwt = p->jw_type % 10;
    const int rtM = (p->bitmask & PFO_RUNTIME_OFFSETM) != 0;
    const int rtV = (p->bitmask & PFO_RUNTIME_OFFSETV) != 0;
    const int64_t oM = p->run_offsetM, oV = p->run_offsetV;
    memset(L, 0, sizeof(*L));
    if (p->upperBanded == 2) {
        /* tridiagonal: ld at 0, md at M, ud at 2M (:117-131).  Only jw_type%10
         * == 3 is defined: with %10 == 2 the bands are loaded only by the
         * matvec (:228-235, :269), so the reference's "solve" is the identity. */
        L->off_md = M; L->off_sl = 0; L->off_su = 2 * M;
        if (jwt == 3) { L->mv = PFO_MV_DIAG; L->sv = PFO_SV_TRI; return 0; }
        return -1;
    }
    if (jwt == 2) L->mv = PFO_MV_NONE;
    else if (jwt == 3) {
        /* jw_type%10 == 3 flips upperBanded while the matvec offsets are
         * chosen (:133-136, :203-206); the matvec is then md-only (:241-245),
         * and the solve reuses the off-diagonal band loaded with it: the solve
         * bands are not reloaded when performTriSolve == 2 (:337-344). */
        L->mv = PFO_MV_DIAG;
        if (p->upperBanded == 1) {
            L->off_md = rtM ? oM : M;
            L->sv = PFO_SV_LOWER;
            L->off_sl = rtM ? oM + M : 0;
        } else {
            L->off_md = rtM ? oM + M : 0;
            L->sv = PFO_SV_UPPER;
            L->off_su = rtM ? oM : M;
        }
        return 0;
    } else if (p->upperBanded == 1) {
        L->mv = PFO_MV_UPPER;
        L->off_md = rtM ? oM + M : 0;
        L->off_mo = rtM ? oM : M;
    } else {
        L->mv = PFO_MV_LOWER;
        L->off_md = rtM ? oM : M;
        L->off_mo = rtM ? oM + M : 0;
    }
    if (jwt == 1) L->sv = PFO_SV_NONE;
    else if (p->upperBanded == 1) { L->sv = PFO_SV_LOWER; L->off_sl = rtV ? oV : 2 * M; }
    else { L->sv = PFO_SV_UPPER; L->off_su = rtV ? oV : 2 * M; }
    return 0;
}

static int64_t band_pos(const pfo_params* p, int64_t i)
{
    return p->bandsPermuted ? pfo_reorder_i0(i, p->M, 0) : i;
}

int pfo_jw_operator(const pfo_params* p, const double* bands, int* mv_kind, int* sv_kind,
                    double* mv_d, double* mv_o, double* sv_l, double* sv_u)
{
    jw_layout L;
    if (jw_resolve(p, &L)) return -1;
    *mv_kind = L.mv; *sv_kind = L.sv;
    for (int64_t i = 0; i < p->M; i++) {
        int64_t k = band_pos(p, i);
        if (L.mv != PFO_MV_NONE && mv_d) mv_d[i] = bands[L.off_md + k];
        if ((L.mv == PFO_MV_UPPER || L.mv == PFO_MV_LOWER) && mv_o) mv_o[i] = bands[L.off_mo + k];
        if ((L.sv == PFO_SV_LOWER || L.sv == PFO_SV_TRI) && sv_l) sv_l[i] = bands[L.off_sl + k];
        if ((L.sv == PFO_SV_UPPER || L.sv == PFO_SV_TRI) && sv_u) sv_u[i] = bands[L.off_su + k];
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* One system in type T: matvec (pfSolve_MatVecMul.h:28-133), unit-diagonal
 * bi-/tridiagonal solve (pfSolve_TridiagonalSolve.h:1578-1929), scaleC on
 * solution row 0 (:1918-1927).  Rows outside [0, M) read as zero, so
 * ld[0] and ud[M-1] never contribute. */
#define DEFINE_SYSTEM(NAME, T)                                                           \
    static void NAME(int mv, int sv, int64_t M, const T* md, const T* mo, const T* sl,   \
                     const T* su, T scaleC, T* b, T* g, T* w)                            \
    {                                                                                    \
        for (int64_t i = 0; i < M; i++) {                                                \
            T v = b[i];                                                                  \
            if (mv == PFO_MV_DIAG) v = md[i] * b[i];                                     \
            else if (mv == PFO_MV_UPPER)                                                 \
                v = md[i] * b[i] + ((i + 1 < M) ? mo[i] * b[i + 1] : (T)0);              \
            else if (mv == PFO_MV_LOWER)                                                 \
                v = md[i] * b[i] + ((i > 0) ? mo[i] * b[i - 1] : (T)0);                  \
            g[i] = v;                                                                    \
        }                                                                                \
        if (sv == PFO_SV_LOWER) {                                                        \
            for (int64_t i = 1; i < M; i++) g[i] = g[i] - sl[i] * g[i - 1];              \
        } else if (sv == PFO_SV_UPPER) {                                                 \
            for (int64_t i = M - 2; i >= 0; i--) g[i] = g[i] - su[i] * g[i + 1];         \
        } else if (sv == PFO_SV_TRI) {                                                   \
            /* Thomas, sample_0_benchmark_VkFFT_single.cpp:437-460, unit diagonal */     \
            w[0] = su[0];                                                                \
            for (int64_t i = 1; i < M; i++) {                                            \
                T den = (T)1 - sl[i] * w[i - 1];                                         \
                w[i] = su[i] / den;                                                      \
                g[i] = (g[i] - sl[i] * g[i - 1]) / den;                                  \
            }                                                                            \
            for (int64_t i = M - 2; i >= 0; i--) g[i] = g[i] - w[i] * g[i + 1];          \
        }                                                                                \
        if (sv != PFO_SV_NONE && M > 0) g[0] = g[0] * scaleC;                            \
    }
DEFINE_SYSTEM(system_q, q_t)
DEFINE_SYSTEM(system_d, double)

typedef struct {
    int64_t offS, oStride;
    int64_t iz0, iz1, oz0, oz1;
    int rtIZ, rtOZ;
    double scaleC;
} rhs_layout;

static void rhs_resolve(const pfo_params* p, rhs_layout* R)
{
    R->offS = rv(p, PFO_RUNTIME_OFFSETSOLUTION, p->cfg_offsetSolution, p->run_offsetSolution);
    R->oStride = rv(p, PFO_RUNTIME_OUTPUTBUFFERSTRIDE, p->cfg_outputBufferStride, p->run_outputBufferStride);
    R->rtIZ = (p->bitmask & PFO_RUNTIME_INPUTZEROPAD) != 0;
    R->rtOZ = (p->bitmask & PFO_RUNTIME_OUTPUTZEROPAD) != 0;
    R->iz0 = R->rtIZ ? p->run_inputZeropad[0] : p->cfg_inputZeropad[0];
    R->iz1 = R->rtIZ ? p->run_inputZeropad[1] : p->cfg_inputZeropad[1];
    R->oz0 = R->rtOZ ? p->run_outputZeropad[0] : p->cfg_outputZeropad[0];
    R->oz1 = R->rtOZ ? p->run_outputZeropad[1] : p->cfg_outputZeropad[1];
    R->scaleC = (p->bitmask & PFO_RUNTIME_SCALEC) ? p->run_scaleC : p->cfg_scaleC;
}

/* Storage kinds for the generic driver. */
enum { ST_F64 = 0, ST_F32 = 1, ST_DD = 2 };

static q_t load_q(const void* a, int st, int64_t k)
{
    if (st == ST_F64) return (q_t)((const double*)a)[k];
    if (st == ST_F32) return (q_t)((const float*)a)[k];
    const double* d = (const double*)a;
    return (q_t)d[2 * k] + (q_t)d[2 * k + 1];
}

static void store_q(void* a, int st, int64_t k, q_t v)
{
    if (st == ST_F64) ((double*)a)[k] = (double)v;
    else if (st == ST_F32) ((float*)a)[k] = (float)v;
    else {
        double hi = (double)v;
        double lo = (double)(v - (q_t)hi);
        ((double*)a)[2 * k] = hi;
        ((double*)a)[2 * k + 1] = lo;
    }
}

static int jw_step_q_generic(const pfo_params* p, const void* bands, void* rhs, int st, int nthreads)
{
    jw_layout L;
    if (jw_resolve(p, &L)) return -1;
    rhs_layout R;
    rhs_resolve(p, &R);
    const int64_t M = p->M;
    q_t* md = (q_t*)calloc((size_t)M + 1, sizeof(q_t));
    q_t* mo = (q_t*)calloc((size_t)M + 1, sizeof(q_t));
    q_t* sl = (q_t*)calloc((size_t)M + 1, sizeof(q_t));
    q_t* su = (q_t*)calloc((size_t)M + 1, sizeof(q_t));
    if (!md || !mo || !sl || !su) { free(md); free(mo); free(sl); free(su); return -1; }
    for (int64_t i = 0; i < M; i++) {
        int64_t k = band_pos(p, i);
        if (L.mv != PFO_MV_NONE) md[i] = load_q(bands, st, L.off_md + k);
        if (L.mv == PFO_MV_UPPER || L.mv == PFO_MV_LOWER) mo[i] = load_q(bands, st, L.off_mo + k);
        if (L.sv == PFO_SV_LOWER || L.sv == PFO_SV_TRI) sl[i] = load_q(bands, st, L.off_sl + k);
        if (L.sv == PFO_SV_UPPER || L.sv == PFO_SV_TRI) su[i] = load_q(bands, st, L.off_su + k);
    }
    q_t sC = (st == ST_F32) ? (q_t)(float)R.scaleC : (q_t)R.scaleC;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        q_t* b = (q_t*)malloc(sizeof(q_t) * (size_t)(M + 1));
        q_t* g = (q_t*)malloc(sizeof(q_t) * (size_t)(M + 1));
        q_t* w = (q_t*)malloc(sizeof(q_t) * (size_t)(M + 1));
#pragma omp for schedule(static)
        for (int64_t y = 0; y < p->batch; y++) {
            int64_t base = R.offS + y * R.oStride;
            for (int64_t i = 0; i < M; i++)
                b[i] = keep(i, R.iz0, R.iz1, R.rtIZ) ? load_q(rhs, st, base + i) : (q_t)0;
            system_q(L.mv, L.sv, M, md, mo, sl, su, sC, b, g, w);
            for (int64_t i = 0; i < M; i++)
                if (keep(i, R.oz0, R.oz1, R.rtOZ)) store_q(rhs, st, base + i, g[i]);
        }
        free(b); free(g); free(w);
    }
    free(md); free(mo); free(sl); free(su);
    return 0;
}

int pfo_jw_step_q(const pfo_params* p, const double* bands, double* rhs, int nthreads)
{
    return jw_step_q_generic(p, bands, rhs, ST_F64, nthreads);
}
int pfo_jw_step_q_f32(const pfo_params* p, const float* bands, float* rhs, int nthreads)
{
    return jw_step_q_generic(p, bands, rhs, ST_F32, nthreads);
}
int pfo_jw_step_q_dd(const pfo_params* p, const double* bands_dd, double* rhs_dd, int nthreads)
{
    return jw_step_q_generic(p, bands_dd, rhs_dd, ST_DD, nthreads);
}

int pfo_jw_step_d(const pfo_params* p, const double* bands, double* rhs, int nthreads)
{
    jw_layout L;
    if (jw_resolve(p, &L)) return -1;
    rhs_layout R;
    rhs_resolve(p, &R);
    const int64_t M = p->M;
    double* md = (double*)calloc((size_t)M + 1, sizeof(double));
    double* mo = (double*)calloc((size_t)M + 1, sizeof(double));
    double* sl = (double*)calloc((size_t)M + 1, sizeof(double));
    double* su = (double*)calloc((size_t)M + 1, sizeof(double));
    if (!md || !mo || !sl || !su) { free(md); free(mo); free(sl); free(su); return -1; }
    for (int64_t i = 0; i < M; i++) {
        int64_t k = band_pos(p, i);
        if (L.mv != PFO_MV_NONE) md[i] = bands[L.off_md + k];
        if (L.mv == PFO_MV_UPPER || L.mv == PFO_MV_LOWER) mo[i] = bands[L.off_mo + k];
        if (L.sv == PFO_SV_LOWER || L.sv == PFO_SV_TRI) sl[i] = bands[L.off_sl + k];
        if (L.sv == PFO_SV_UPPER || L.sv == PFO_SV_TRI) su[i] = bands[L.off_su + k];
    }
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        double* b = (double*)malloc(sizeof(double) * (size_t)(M + 1));
        double* g = (double*)malloc(sizeof(double) * (size_t)(M + 1));
        double* w = (double*)malloc(sizeof(double) * (size_t)(M + 1));
#pragma omp for schedule(static)
        for (int64_t y = 0; y < p->batch; y++) {
            int64_t base = R.offS + y * R.oStride;
            for (int64_t i = 0; i < M; i++) b[i] = keep(i, R.iz0, R.iz1, R.rtIZ) ? rhs[base + i] : 0.0;
            system_d(L.mv, L.sv, M, md, mo, sl, su, R.scaleC, b, g, w);
            for (int64_t i = 0; i < M; i++)
                if (keep(i, R.oz0, R.oz1, R.rtOZ)) rhs[base + i] = g[i];
        }
        free(b); free(g); free(w);
    }
    free(md); free(mo); free(sl); free(su);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* ALT stride-2 mode (jw_type / 100 % 10 == 1, pfSolve_Plan_JonesWorland.h:265).
 * The kernel's lanes split in two halves (pfSolve_TridiagonalSolve.h:1319-1330
 * read, :1475-1486 write, :1622-1644 solve): lane t < T/2 holds the even rows
 * 2 (t R + i), lane t >= T/2 the odd rows 2 ((t - T/2) R + i) + 1, i < R, with
 * T lanes and R = ceil(M / T) rows per lane as for any JW plan.  The matvec
 * couples register i with i + 1 (rows r and r + 2) and each half solves its
 * own parity, so rows of one parity form an independent system with
 * neighbours r -+ 2.  Band entries of every register are loaded with all
 * lanes active (pfSolve_ReadWrite.h:1637-1645, 1705-1711): the entry of row r
 * sits at position i T + t, and the bands are R T entries apart instead of M
 * (pfSolve_JonesWorland.h:209-222, 262-271).  scaleC multiplies row 0 only
 * (lane 0 after the halves are merged again, :1901-1927). */
static void alt_geometry(int64_t M, int64_t* T, int64_t* R)
{
    int64_t warp = 64 * ((M + 1023) / 1024);
    if (M < 512) warp = 32;
    if (warp < 32) warp = 32;
    if (warp % 32) warp = 32 * ((warp + 31) / 32);
    *T = warp;
    *R = (M + warp - 1) / warp;
}

int64_t pfo_alt_position(int64_t r, int64_t M)
{
    int64_t T, R;
    alt_geometry(M, &T, &R);
    const int64_t h = r & 1, e = r >> 1;
    const int64_t t = h * (T / 2) + e / R, i = e % R;
    return i * T + t;
}

int pfo_jw_step_alt_q(const pfo_params* p, const double* bands, double* rhs, int nthreads)
{
    if (((p->jw_type / 100) % 10) != 1) return -1;
    if (p->bitmask & (PFO_RUNTIME_OFFSETM | PFO_RUNTIME_OFFSETV)) return -1;
    int64_t T, R;
    alt_geometry(p->M, &T, &R);
    pfo_params q = *p;
    q.M = R * T;  /* band offsets: multiples of R T */
    jw_layout L;
    if (jw_resolve(&q, &L)) return -1;
    rhs_layout RL;
    rhs_resolve(p, &RL);
    const int64_t M = p->M;
    q_t* co = (q_t*)calloc((size_t)(4 * (M + 2)), sizeof(q_t));
    if (!co) return -1;
    q_t *md = co, *mo = co + (M + 2), *sl = co + 2 * (M + 2), *su = co + 3 * (M + 2);
    for (int64_t r = 0; r < M; r++) {
        const int64_t k = pfo_alt_position(r, M);
        if (L.mv != PFO_MV_NONE) md[r] = (q_t)bands[L.off_md + k];
        if (L.mv == PFO_MV_UPPER || L.mv == PFO_MV_LOWER) mo[r] = (q_t)bands[L.off_mo + k];
        if (L.sv == PFO_SV_LOWER || L.sv == PFO_SV_TRI) sl[r] = (q_t)bands[L.off_sl + k];
        if (L.sv == PFO_SV_UPPER || L.sv == PFO_SV_TRI) su[r] = (q_t)bands[L.off_su + k];
    }
    const q_t sC = (q_t)RL.scaleC;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        const int64_t Mh = (M + 1) / 2 + 1;
        q_t* b = (q_t*)malloc(sizeof(q_t) * (size_t)Mh);
        q_t* g = (q_t*)malloc(sizeof(q_t) * (size_t)Mh);
        q_t* w = (q_t*)malloc(sizeof(q_t) * (size_t)Mh);
        q_t* c4 = (q_t*)malloc(sizeof(q_t) * (size_t)(4 * Mh));
#pragma omp for schedule(static)
        for (int64_t y = 0; y < p->batch; y++) {
            const int64_t base = RL.offS + y * RL.oStride;
            for (int h = 0; h < 2; h++) {
                const int64_t n = (M - h + 1) / 2;  /* rows of this parity */
                if (n <= 0) continue;
                for (int64_t e = 0; e < n; e++) {
                    const int64_t r = 2 * e + h;
                    b[e] = keep(r, RL.iz0, RL.iz1, RL.rtIZ) ? (q_t)rhs[base + r] : (q_t)0;
                    c4[e] = md[r];
                    c4[Mh + e] = mo[r];
                    c4[2 * Mh + e] = sl[r];
                    c4[3 * Mh + e] = su[r];
                }
                system_q(L.mv, L.sv, n, c4, c4 + Mh, c4 + 2 * Mh, c4 + 3 * Mh, h == 0 ? sC : (q_t)1, b, g, w);
                for (int64_t e = 0; e < n; e++) {
                    const int64_t r = 2 * e + h;
                    if (keep(r, RL.oz0, RL.oz1, RL.rtOZ)) rhs[base + r] = (double)g[e];
                }
            }
        }
        free(b); free(g); free(w); free(c4);
    }
    free(co);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* K consecutive JW steps in one kernel (numConsecutiveJWIterations = K > 1;
 * pfSolve_KernelsLevel2/pfSolve_JonesWorland.h:108-374).
 *
 *  - Step s works on M_s = M - s rows (upperBanded 1 or 2) or M + s rows
 *    (upperBanded 0) (:109-115).  The right-hand side is read once with M rows
 *    (rows beyond stay zero, pfSolve_Registers.h:171-177) and written once with
 *    M_{K-1} rows (pfSolve_ReadWrite.h:1934-1935 with the final M_size);
 *    rows in between stay in registers, so a row that leaves the system keeps
 *    its last value and is not written back.
 *  - Bands of step s come from buffer s when there are several input buffers
 *    (pfSolve_Transfers.h:250-265), else from buffer 0, at offsets that depend
 *    on M_s (:117-207, :269-353), in register-major order for M_s rows with the
 *    register count of the plan (computed from M + K - 1 for upperBanded 0,
 *    pfSolve_Plan_JonesWorland.h:276-283, 342-346).  Rows at or beyond M_s
 *    read md = 1, ld = ud = 0 (pfSolve_ReadWrite.h:1678-1695).
 *  - The matvec diagonal is applied at the first step (upperBanded 1) or the
 *    last (upperBanded 0) only (pfSolve_MatVecMul.h:74-75, 98-101); for
 *    upperBanded 2 the diagonal is reloaded only at steps 0 and K-1
 *    (pfSolve_ReadWrite.h:1650), so only K = 2 is defined there.  jw_type%10
 *    == 3 with upperBanded 0/1 multiplies by a diagonal that is not reloaded
 *    for K > 1 and is rejected.
 *  - The off-diagonal entry of row M_s - 1 couples to row M_s, which still
 *    holds a value after a shrinking step; scaleC multiplies solution row 0
 *    after every solve (pfSolve_TridiagonalSolve.h:1918-1927). */
static int64_t reorder_r(int64_t i, int64_t M, int64_t r)
{
    int64_t t = i / r, j = i % r;
    int64_t m = M % r, ceil_n = (M + r - 1) / r, floor_n = M / r;
    return t + ((j < m) ? j * ceil_n : m * ceil_n + (j - m) * floor_n);
}

int64_t pfo_steps_registers(int64_t M, int upperBanded, int K)
{
    int64_t tempM = upperBanded ? M : M + K - 1;
    int64_t warp = 64 * ((tempM + 1023) / 1024);
    if (tempM < 512) warp = 32;
    if (warp < 32) warp = 32;
    if (warp % 32) warp = 32 * ((warp + 31) / 32);
    int64_t r = (tempM + warp - 1) / warp;
    return r < 1 ? 1 : r;
}

int pfo_jw_steps_layout(const pfo_params* p, int K, int s, pfo_step* st)
{
    const int ub = p->upperBanded, jwt = p->jw_type % 10;
    if (K < 1 || s < 0 || s >= K) return -1;
    if (ub == 2 && (jwt != 3 || K > 2)) return -1;
    if (ub != 2 && (jwt == 3 || (jwt != 0 && jwt != 1 && jwt != 2))) return -1;
    const int rtM = (p->bitmask & PFO_RUNTIME_OFFSETM) != 0;
    const int rtV = (p->bitmask & PFO_RUNTIME_OFFSETV) != 0;
    const int64_t oM = p->run_offsetM, oV = p->run_offsetV;
    const int64_t Ms = ub ? p->M - s : p->M + s;
    if (Ms < 1) return -1;
    memset(st, 0, sizeof(*st));
    st->M = Ms;
    st->r = pfo_steps_registers(p->M, ub, K);
    if (ub == 2) {
        st->mv = PFO_MV_DIAG; st->diag = 1; st->off_md = Ms;
        st->sv = PFO_SV_TRI; st->off_sl = 0; st->off_su = 2 * Ms;
        return 0;
    }
    if (jwt != 2) {
        if (ub == 1) {
            st->mv = PFO_MV_UPPER; st->diag = (s == 0);
            st->off_md = rtM ? oM + Ms : 0;
            st->off_mo = rtM ? oM : (s == 0 ? Ms : 0);
        } else {
            st->mv = PFO_MV_LOWER; st->diag = (s == K - 1);
            st->off_md = rtM ? oM : Ms;
            st->off_mo = rtM ? oM + Ms : 0;
        }
    }
    if (jwt != 1) {
        if (ub == 1) { st->sv = PFO_SV_LOWER; st->off_sl = rtV ? oV : (s == 0 ? 2 * Ms : Ms); }
        else { st->sv = PFO_SV_UPPER; st->off_su = rtV ? oV : (s == K - 1 ? 2 * Ms : Ms); }
    }
    return 0;
}

#define DEFINE_STEPS(NAME, T)                                                                           \
    int NAME(const pfo_params* p, int K, int nbuf, const double* const* bands, double* rhs, int nthreads) \
    {                                                                                                   \
        if (K < 2 || K > PFO_MAX_STEPS || (nbuf != 1 && nbuf < K) || !bands) return -1;                \
        pfo_step st[PFO_MAX_STEPS];                                                                     \
        for (int s = 0; s < K; s++)                                                                     \
            if (pfo_jw_steps_layout(p, K, s, &st[s])) return -1;                                       \
        rhs_layout R;                                                                                   \
        rhs_resolve(p, &R);                                                                             \
        const int64_t M0 = p->M, Mout = st[K - 1].M;                                                    \
        const int64_t total = (M0 > Mout ? M0 : Mout) + 1;                                              \
        T* co = (T*)calloc((size_t)(4 * K * total), sizeof(T));                                         \
        if (!co) return -1;                                                                             \
        for (int s = 0; s < K; s++) {                                                                   \
            const double* b = bands[nbuf > 1 ? s : 0];                                                  \
            T* md = co + (4 * s + 0) * total;                                                           \
            T* mo = co + (4 * s + 1) * total;                                                           \
            T* sl = co + (4 * s + 2) * total;                                                           \
            T* su = co + (4 * s + 3) * total;                                                           \
            for (int64_t i = 0; i < st[s].M; i++) {                                                     \
                const int64_t k = p->bandsPermuted ? reorder_r(i, st[s].M, st[s].r) : i;                \
                md[i] = (st[s].mv != PFO_MV_NONE && st[s].diag) ? (T)b[st[s].off_md + k] : (T)1;        \
                if (st[s].mv == PFO_MV_UPPER || st[s].mv == PFO_MV_LOWER) mo[i] = (T)b[st[s].off_mo + k]; \
                if (st[s].sv == PFO_SV_LOWER || st[s].sv == PFO_SV_TRI) sl[i] = (T)b[st[s].off_sl + k]; \
                if (st[s].sv == PFO_SV_UPPER || st[s].sv == PFO_SV_TRI) su[i] = (T)b[st[s].off_su + k]; \
            }                                                                                           \
        }                                                                                               \
        const T sC = (T)R.scaleC;                                                                       \
        _Pragma("omp parallel num_threads(nthreads > 0 ? nthreads : 1)")                                \
        {                                                                                               \
            T* x = (T*)malloc(sizeof(T) * (size_t)total);                                               \
            T* y = (T*)malloc(sizeof(T) * (size_t)total);                                               \
            T* w = (T*)malloc(sizeof(T) * (size_t)total);                                               \
            _Pragma("omp for schedule(static)")                                                         \
            for (int64_t q = 0; q < p->batch; q++) {                                                    \
                const int64_t base = R.offS + q * R.oStride;                                            \
                for (int64_t i = 0; i < total; i++)                                                     \
                    x[i] = (i < M0 && keep(i, R.iz0, R.iz1, R.rtIZ)) ? (T)rhs[base + i] : (T)0;         \
                for (int s = 0; s < K; s++) {                                                           \
                    const int64_t Ms = st[s].M;                                                         \
                    const T* md = co + (4 * s + 0) * total;                                             \
                    const T* mo = co + (4 * s + 1) * total;                                             \
                    const T* sl = co + (4 * s + 2) * total;                                             \
                    const T* su = co + (4 * s + 3) * total;                                             \
                    for (int64_t i = 0; i < total; i++) y[i] = x[i];                                    \
                    if (st[s].mv != PFO_MV_NONE)                                                        \
                        for (int64_t i = 0; i < Ms; i++) {                                              \
                            T v = md[i] * x[i];                                                         \
                            if (st[s].mv == PFO_MV_UPPER) v += mo[i] * x[i + 1];                        \
                            if (st[s].mv == PFO_MV_LOWER && i > 0) v += mo[i] * x[i - 1];               \
                            y[i] = v;                                                                   \
                        }                                                                               \
                    if (st[s].sv == PFO_SV_LOWER) {                                                     \
                        for (int64_t i = 1; i < Ms; i++) y[i] = y[i] - sl[i] * y[i - 1];                \
                    } else if (st[s].sv == PFO_SV_UPPER) {                                              \
                        for (int64_t i = Ms - 1; i >= 0; i--) y[i] = y[i] - su[i] * y[i + 1];           \
                    } else if (st[s].sv == PFO_SV_TRI) {                                                \
                        /* rows 0..Ms: row Ms is an identity row coupled from above */                  \
                        w[0] = su[0];                                                                   \
                        for (int64_t i = 1; i <= Ms; i++) {                                             \
                            const T a = (i < Ms) ? sl[i] : (T)0;                                        \
                            const T c = (i < Ms) ? su[i] : (T)0;                                        \
                            const T den = (T)1 - a * w[i - 1];                                          \
                            w[i] = c / den;                                                             \
                            y[i] = (y[i] - a * y[i - 1]) / den;                                         \
                        }                                                                               \
                        for (int64_t i = Ms - 1; i >= 0; i--) y[i] = y[i] - w[i] * y[i + 1];            \
                    }                                                                                   \
                    if (st[s].sv != PFO_SV_NONE) y[0] = y[0] * sC;                                      \
                    for (int64_t i = 0; i < total; i++) x[i] = y[i];                                    \
                }                                                                                       \
                for (int64_t i = 0; i < Mout; i++)                                                      \
                    if (keep(i, R.oz0, R.oz1, R.rtOZ)) rhs[base + i] = (double)x[i];                    \
            }                                                                                           \
            free(x); free(y); free(w);                                                                  \
        }                                                                                               \
        free(co);                                                                                       \
        return 0;                                                                                       \
    }
DEFINE_STEPS(pfo_jw_steps_q, q_t)
DEFINE_STEPS(pfo_jw_steps_d, double)

/* ------------------------------------------------------------------------- */
/* dgbmv: y_r = sum_j A[offsetM + j*M + c] x_c, c = r + KU - j, 0 <= c < M
 * (pfSolve_MatVecMul.h:389-443).  The plan-time offsetM is honoured here
 * (pfSolve_dgbmv.h:79-87), unlike the JW kernel. */
/* ALT_dgbmv (pfSolve_Plan_dgbmv.h:100, pfSolve_MatVecMul.h:390): band j is
 * dropped when (j % 2 == 1 - LDA % 2 and KL != 0) or (j % 2 == LDA % 2 and
 * KU != 0), KL and KU as configured.  With one side only and KU, or KL odd,
 * this keeps the couplings at even distance; the rule is restated as written. */
int pfo_dgbmv_band_dropped(const pfo_params* p, int64_t j)
{
    if (!p->ALT_dgbmv) return 0;
    const int64_t par = p->LDA % 2;
    return ((j % 2) == 1 - par && p->KL) || ((j % 2) == par && p->KU);
}

#define DEFINE_DGBMV(NAME, T)                                                              \
    int NAME(const pfo_params* p, const double* A, double* rhs, int nthreads)              \
    {                                                                                      \
        rhs_layout R;                                                                      \
        rhs_resolve(p, &R);                                                                \
        const int64_t M = p->M;                                                            \
        const int64_t offM = rv(p, PFO_RUNTIME_OFFSETM, p->cfg_offsetM, p->run_offsetM);   \
        if (p->LDA <= 0 || p->KU < 0 || p->KU >= p->LDA) return -1;                        \
        _Pragma("omp parallel num_threads(nthreads > 0 ? nthreads : 1)")                   \
        {                                                                                  \
            T* x = (T*)malloc(sizeof(T) * (size_t)(M + 1));                                \
            _Pragma("omp for schedule(static)")                                            \
            for (int64_t y = 0; y < p->batch; y++) {                                       \
                int64_t base = R.offS + y * R.oStride;                                     \
                for (int64_t i = 0; i < M; i++)                                            \
                    x[i] = keep(i, R.iz0, R.iz1, R.rtIZ) ? (T)rhs[base + i] : (T)0;        \
                for (int64_t r = 0; r < M; r++) {                                          \
                    T acc = 0;                                                             \
                    for (int64_t j = 0; j < p->LDA; j++) {                                 \
                        int64_t c = r + p->KU - j;                                         \
                        if (c < 0 || c >= M || pfo_dgbmv_band_dropped(p, j)) continue;     \
                        acc += (T)A[offM + j * M + c] * x[c];                              \
                    }                                                                      \
                    if (keep(r, R.oz0, R.oz1, R.rtOZ)) rhs[base + r] = (double)acc;        \
                }                                                                          \
            }                                                                              \
            free(x);                                                                       \
        }                                                                                  \
        return 0;                                                                          \
    }
DEFINE_DGBMV(pfo_dgbmv_q, q_t)
DEFINE_DGBMV(pfo_dgbmv_d, double)

/* ------------------------------------------------------------------------- */
/* Scale operators, runtime-scaleC branch (pfSolve_RegistersScaleC.h:27-201);
 * x is the row index inside the system, L = lshift, s = scaleC. */
static q_t scale_factor_q(int kind, int64_t x, int L, q_t s)
{
    q_t X = (q_t)x;
    switch (kind) {
    case 1: return s;
    case 2: return (q_t)2 * (X + L + 1) * sqrtq((X + 1) / (X + s + L + (q_t)1.5));
    case 3:
        return (q_t)4 * (X + L + 2) * (X + L + 3) *
               sqrtq((X + 1) * (X + 2) / ((X + s + L + (q_t)2.5) * (X + s + L + (q_t)3.5)));
    case 4: return ((q_t)4 * L + 6) * (X + L + 1) * sqrtq((X + 1) / (X + s + L + (q_t)1.5));
    default: return (q_t)1;
    }
}

double pfo_scale_factor(int kind, int64_t x, int lshift, double s)
{
    return (double)scale_factor_q(kind, x, lshift, (q_t)s);
}

/* Block kernel: element (x = e mod size0, y = e div size0); read at
 * offsetM + y*inputStride + x, write at offsetSolution + y*outputStride + x
 * (pfSolve_ReadWrite.h:2293-2317).  block%10 picks the layout conversion
 * (XXII = per-row real block then imaginary block, pfSolve_ReadWrite.h:2313-2354,
 * with the in/out types of pfSolve_KernelStartEnd.h:1089-1097), block/10%10 == 2
 * accumulates into the output (:2320-2329), block/100 picks the Scale
 * operator.  Scale operators multiply both components of a complex value by
 * the real factor.  block/100 == 1 with a plan-time scaleC of 0 writes zeros
 * without reading (pfSolve_block.h:82). */
int pfo_block_q(const pfo_params* p, const double* in, double* out)
{
    const int bt = p->block % 10, acc = ((p->block / 10) % 10) == 2, sk = p->block / 100;
    if (bt < 1 || bt > 7 || sk > 4) return -1;
    if (acc && bt == 4) return -1; /* reads a real into a complex register: undefined */
    rhs_layout R;
    rhs_resolve(p, &R);
    const int64_t offM = rv(p, PFO_RUNTIME_OFFSETM, p->cfg_offsetM, p->run_offsetM);
    const int64_t iS = rv(p, PFO_RUNTIME_INPUTBUFFERSTRIDE, p->cfg_inputBufferStride, p->run_inputBufferStride);
    const int64_t oS = R.oStride, offS = R.offS;
    const int rtC = (p->bitmask & PFO_RUNTIME_SCALEC) != 0;
    const int skip = (sk == 1) && !rtC && (p->cfg_scaleC == 0.0);
    const q_t s = (q_t)R.scaleC;
    for (int64_t y = 0; y < p->size1; y++) {
        for (int64_t x = 0; x < p->size0; x++) {
            q_t vr = 0, vi = 0;
            if (!skip) {
                if (keep(x, R.iz0, R.iz1, R.rtIZ)) {
                    int64_t ii = offM + y * iS;
                    switch (bt) {
                    case 1: vr = in[ii + x]; break;
                    case 2: case 3: case 4: vr = in[2 * (ii + x)]; vi = in[2 * (ii + x) + 1]; break;
                    case 5: vr = in[ii + x]; break;
                    case 6: vi = in[ii + x]; break;
                    case 7: vr = in[2 * ii + x]; vi = in[2 * ii + x + iS]; break;
                    }
                }
                if (sk) {
                    q_t f = scale_factor_q(sk, x, p->lshift, s);
                    vr *= f; vi *= f;
                }
            }
            if (!keep(x, R.oz0, R.oz1, R.rtOZ)) continue;
            int64_t oi = offS + y * oS;
            switch (bt) {
            case 1: case 2:
                if (acc) vr += out[oi + x];
                out[oi + x] = (double)vr;
                break;
            case 3:
                if (acc) vi += out[oi + x];
                out[oi + x] = (double)vi;
                break;
            case 4:
                out[2 * oi + x] = (double)vr;
                out[2 * oi + x + oS] = (double)vi;
                break;
            default:
                if (acc) { vr += out[2 * (oi + x)]; vi += out[2 * (oi + x) + 1]; }
                out[2 * (oi + x)] = (double)vr;
                out[2 * (oi + x) + 1] = (double)vi;
                break;
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
void pfo_rel_errors(const double* a, const double* ref, int64_t M, int64_t batch, int64_t stride,
                    int64_t offset, double* rel_l2_max, double* rel_max)
{
    double worst_l2 = 0, dmax = 0, rmax = 0;
    for (int64_t y = 0; y < batch; y++) {
        const double* pa = a + offset + y * stride;
        const double* pr = ref + offset + y * stride;
        q_t num = 0, den = 0;
        for (int64_t i = 0; i < M; i++) {
            q_t d = (q_t)pa[i] - (q_t)pr[i];
            num += d * d;
            den += (q_t)pr[i] * (q_t)pr[i];
            double ad = fabs((double)d), ar = fabs(pr[i]);
            if (ad > dmax) dmax = ad;
            if (ar > rmax) rmax = ar;
        }
        double e = (den > 0) ? (double)sqrtq(num / den) : (double)sqrtq(num);
        if (e > worst_l2) worst_l2 = e;
    }
    *rel_l2_max = worst_l2;
    *rel_max = (rmax > 0) ? dmax / rmax : dmax;
}

/* Relative errors for double-double storage ({hi, lo} pairs), in __float128. */
void pfo_rel_errors_dd(const double* a, const double* ref, int64_t M, int64_t batch, int64_t stride,
                       int64_t offset, double* rel_l2_max, double* rel_max)
{
    double worst = 0, dmax = 0, rmax = 0;
    for (int64_t y = 0; y < batch; y++) {
        q_t num = 0, den = 0;
        for (int64_t i = 0; i < M; i++) {
            const int64_t k = offset + y * stride + i;
            const q_t va = (q_t)a[2 * k] + (q_t)a[2 * k + 1];
            const q_t vr = (q_t)ref[2 * k] + (q_t)ref[2 * k + 1];
            const q_t d = va - vr;
            num += d * d;
            den += vr * vr;
            const double ad = fabs((double)d), ar = fabs((double)vr);
            if (ad > dmax) dmax = ad;
            if (ar > rmax) rmax = ar;
        }
        const double e = (den > 0) ? (double)sqrtq(num / den) : (double)sqrtq(num);
        if (e > worst) worst = e;
    }
    *rel_l2_max = worst;
    *rel_max = (rmax > 0) ? dmax / rmax : dmax;
}

/* ---- DCT step (see jw_oracle.h). */
int pfo_dct_q(int type, int64_t N, int64_t nsys, const double* in, int64_t in_stride, double* out,
              int64_t out_stride, int nthreads)
{
    if ((type != 2 && type != 3) || N < 1) return -1;
    /* c[j] = cos(pi j / (2N)), j in [0, 4N) */
    q_t* c = (q_t*)malloc(sizeof(q_t) * 4 * N);
    if (!c) return -1;
    const q_t pi = M_PIq;
    for (int64_t j = 0; j < 4 * N; j++) c[j] = cosq(pi * (q_t)j / (q_t)(2 * N));
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(static)
    for (int64_t y = 0; y < nsys; y++) {
        const double* x = in + y * in_stride;
        double* X = out + y * out_stride;
        for (int64_t k = 0; k < N; k++) {
            q_t acc = 0;
            if (type == 2) {
                for (int64_t n = 0; n < N; n++) acc += (q_t)x[n] * c[(k * (2 * n + 1)) % (4 * N)];
                acc *= 2;
            } else {
                for (int64_t n = 1; n < N; n++) acc += (q_t)x[n] * c[(n * (2 * k + 1)) % (4 * N)];
                acc = 2 * acc + (q_t)x[0];
            }
            X[k] = (double)acc;
        }
    }
    free(c);
    return 0;
}
