// dct.cuh -- the radial DCT step that feeds the JW chain: batched real DCT-II
// and DCT-III of rows of N = 2^p points (8 <= N <= 4096), FP64.
//
// Definitions (FFTW's unnormalized REDFT10 / REDFT01, which the VkFFT that
// PfSolve carries performDCT from follows; pfSolve_Structs.h:272):
//   type 2: X_k = 2 sum_{n} x_n cos(pi k (2n+1) / (2N))
//   type 3: x_k = X_0 + 2 sum_{n>=1} X_n cos(pi n (2k+1) / (2N))
// Both run through a complex N-point FFT (Makhoul, IEEE TASSP 28 (1980)):
//   type 2: v = (x_0, x_2, ..., x_{N-2}, x_{N-1}, ..., x_3, x_1), V = FFT(v),
//           X_k = 2 Re(e^{-i pi k/2N} V_k);
//   type 3: z_k = e^{-i pi k/2N} (X_k + i X_{N-k}) (X_N = 0), Z = FFT(z),
//           x_{2n} = Re Z_n, x_{2n+1} = Re Z_{N-1-n}
// (type 3 is the inverse transform of the conjugate sequence; the real part
// of the conjugate is that of Z).
//
// The FFT is Stockham's self-sorting form in shared memory, in place (each
// stage reads, synchronises, writes): radix-8 stages, then one radix-4 or
// radix-2 stage when log2 N is not a multiple of 3; every thread does one
// radix-8 butterfly per stage (N/8 threads per row), and a CTA holds as many
// row pairs as 256 threads cover: one FFT transforms two rows (see the
// kernel).  Each thread loads the next pair's inputs into registers while the
// current pair is transformed.  Twiddles e^{-2 pi i j/N} and the
// pre/post factors (cos, sin)(pi k/2N) come from tables the plan computes once
// in long double on the host.  Rows are read and written with coalesced
// global accesses; a row is fully staged before its result is written, so
// the transform may run in place.  The step is bound by HBM bandwidth at
// large batches (16 bytes moved per point, in and out).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "jw_types.h"

namespace pfb {

template <int LOGN>
struct DctShape {
    static constexpr int N = 1 << LOGN;
    static constexpr int TPS = N >= 8 ? N / 8 : 1;    // threads per row
    static constexpr int NT = TPS > 256 ? TPS : 256;  // threads per CTA
    static constexpr int SPC = NT / TPS;              // row pairs per CTA round
    static constexpr int L8 = LOGN / 3;               // radix-8 stages
    static constexpr int REM = LOGN % 3;              // then one radix-2 (1) or radix-4 (2) stage
    static constexpr int NP = N + N / 8;  // the buffer, one 16-byte pad after every 8 values
    static constexpr int NTW = N + N / 8 + N / 64 + 1;  // the twiddles, padded (dct_twpad)
    // one buffer of N complex values per row pair, then the twiddles
    static constexpr size_t SMEM = ((size_t)SPC * NP + NTW) * 16;
};

__device__ __forceinline__ double2 dct_cmul(double2 a, double2 b)
{
    return make_double2(__fma_rn(a.x, b.x, -a.y * b.y), __fma_rn(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 dct_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 dct_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// times -i
__device__ __forceinline__ double2 dct_mi(double2 a) { return make_double2(a.y, -a.x); }

template <int R>
__device__ __forceinline__ void dct_dft(double2 (&a)[R]);

template <>
__device__ __forceinline__ void dct_dft<2>(double2 (&a)[2])
{
    const double2 t = a[0];
    a[0] = dct_add(t, a[1]);
    a[1] = dct_sub(t, a[1]);
}

template <>
__device__ __forceinline__ void dct_dft<4>(double2 (&a)[4])
{
    const double2 t0 = dct_add(a[0], a[2]), t1 = dct_sub(a[0], a[2]);
    const double2 t2 = dct_add(a[1], a[3]), t3 = dct_mi(dct_sub(a[1], a[3]));
    a[0] = dct_add(t0, t2);
    a[1] = dct_add(t1, t3);
    a[2] = dct_sub(t0, t2);
    a[3] = dct_sub(t1, t3);
}

// Radix 8 by one decimation-in-frequency step into two radix-4 transforms:
// the first gives the even outputs, the second (after the e^{-2 pi i r/8}
// twiddles) the odd ones.
template <>
__device__ __forceinline__ void dct_dft<8>(double2 (&a)[8])
{
    constexpr double h = 0.70710678118654752440;  // sqrt(2)/2
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const double2 t = a[r];
        a[r] = dct_add(t, a[r + 4]);
        a[r + 4] = dct_sub(t, a[r + 4]);
    }
    a[5] = make_double2(h * (a[5].x + a[5].y), h * (a[5].y - a[5].x));    // e^{-i pi/4}
    a[6] = dct_mi(a[6]);                                                  // e^{-i pi/2}
    a[7] = make_double2(h * (a[7].y - a[7].x), -h * (a[7].x + a[7].y));   // e^{-3 i pi/4}
    double2 f[4] = {a[0], a[1], a[2], a[3]}, g[4] = {a[4], a[5], a[6], a[7]};
    dct_dft<4>(f);
    dct_dft<4>(g);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        a[2 * m] = f[m];
        a[2 * m + 1] = g[m];
    }
}

// Position of value i in a row's buffer: one 16-byte pad after every 8 values,
// so that a first-stage butterfly's 8 consecutive outputs (thread b writes
// 8b .. 8b+7) fall on different banks from its neighbours'.
__device__ __forceinline__ int dct_pad(int i) { return i + (i >> 3); }
// Position of twiddle i in the CTA's table: a stage reads it at a stride of
// N/(Ns R) (1 to 64), and with one pad after every 8 and another after every
// 64 values, the 8 threads of a 16-byte access phase land on 8 different
// bank groups at each of those strides.
__device__ __forceinline__ int dct_twpad(int i) { return i + (i >> 3) + (i >> 6); }

// One Stockham stage of radix R over N points with Ns points already
// transformed per sub-sequence, in place: butterfly b reads buf[b + r N/R],
// twiddles by e^{-2 pi i r k/(Ns R)} (k = b mod Ns), and, once every thread
// of the row has read (`sync`), writes buf[(b - k) R + k + r Ns].  With
// MAKHOUL_IN the buffer holds the rows in their natural order and the stage
// reads sequence point p from Makhoul's position of it (2p for p < N/2,
// 2N - 1 - 2p above); with OUT = 1 the stage writes point q there, so the
// result leaves in the natural order.  Either way the reordering costs no
// pass of its own, and both halves touch 8 different bank groups per access
// phase.  OUT = 2 writes the natural order without the pads: type 2's last
// stage, so that the post-processing's reads of Z_k and Z_{N-k} (ascending
// and descending runs of 8) each touch 8 different bank groups.
template <int R, int N, int TPS, bool MAKHOUL_IN = false, int OUT = 0, class SY>
__device__ __forceinline__ void dct_stage(double2* buf, int Ns, int j, const double2* tw, SY sync)
{
    constexpr int NBF = N / R, NB = NBF / TPS;
    double2 a[NB][R];
#pragma unroll
    for (int i = 0; i < NB; ++i)
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int p = j + i * TPS + r * NBF;
            a[i][r] = buf[dct_pad(MAKHOUL_IN ? (p < N / 2 ? 2 * p : 2 * N - 1 - 2 * p) : p)];
        }
    sync();
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const int b = j + i * TPS;
        const int k = b & (Ns - 1);
        if (Ns > 1) {
            // w^r for r = 1 .. R-1 from w = e^{-2 pi i k/(Ns R)} (one table
            // value, then products: the error grows by about an ulp a factor)
            double2 wr[R];
            wr[1] = tw[dct_twpad(k * (N / (Ns * R)))];
#pragma unroll
            for (int r = 2; r < R; ++r) wr[r] = dct_cmul(wr[r / 2], wr[r - r / 2]);
#pragma unroll
            for (int r = 1; r < R; ++r) a[i][r] = dct_cmul(a[i][r], wr[r]);
        }
        dct_dft<R>(a[i]);
        const int base = (b - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int q = base + r * Ns;
            if constexpr (OUT == 2) buf[q] = a[i][r];
            else buf[dct_pad(OUT == 1 ? (q < N / 2 ? 2 * q : 2 * N - 1 - 2 * q) : q)] = a[i][r];
        }
    }
    sync();
}

// tw[j] = e^{-2 pi i j/N} (j < N); pt[k] = (cos, sin)(pi k/(2N)) (k < N).
//
// Two rows share one complex FFT (a "pair"; rows 2u and 2u + 1):
//   type 2: c = v1 + i v2 (both rows in Makhoul's order), Z = FFT(c); with
//           Zr = Z_{N-k} (Z_0 for k = 0) the rows' transforms are
//           X1_k = (Re Z + Re Zr) cos t + (Im Z - Im Zr) sin t,
//           X2_k = (Im Z + Im Zr) cos t - (Re Z - Re Zr) sin t   (t = pi k/2N);
//   type 3: each row's z_k = e^{-i t}(X_k + i X_{N-k}) is conjugate-symmetric
//           (z_{N-k} = conj z_k), so FFT(z) is real: c = z1 + i z2 gives
//           Re FFT(c) = FFT(z1) and Im FFT(c) = FFT(z2).
// One buffer of N complex values per pair; each thread keeps the next pair's
// 2 N/TPS input values in registers, loaded while the current pair is
// transformed.
template <int LOGN, int TYPE>
__global__ void __launch_bounds__(DctShape<LOGN>::NT, DctShape<LOGN>::NT <= 256 ? 2 : 1)
    dct_kernel(const DctIO io, const double2* __restrict__ tw, const double2* __restrict__ pt)
{
    using S = DctShape<LOGN>;
    constexpr int N = S::N, TPS = S::TPS, PER = N / TPS;
    extern __shared__ __align__(16) double2 dct_smem[];
    const int s = threadIdx.x / TPS, j = threadIdx.x - s * TPS;
    double2* buf = dct_smem + (size_t)s * S::NP;
    double2* tws = dct_smem + (size_t)S::SPC * S::NP;  // the twiddles, shared by the CTA's pairs
    for (int i = threadIdx.x; i < N; i += blockDim.x) tws[dct_twpad(i)] = __ldg(&tw[i]);
    __syncthreads();
    // The threads of one pair synchronise among themselves only: a warp
    // (pairs of up to 256 points share warps, and keep in step), else a named
    // barrier per pair (ids 1..SPC).
    auto sync = [&]() {
        if constexpr (TPS <= 32) __syncwarp();
        else asm volatile("bar.sync %0, %1;\n" ::"r"(1 + s), "r"(TPS) : "memory");
    };
    const int64_t npairs = (io.nsys + 1) / 2;
    const int64_t stride_units = (int64_t)gridDim.x * S::SPC;
    double p1[PER], p2[PER];
    auto fetch = [&](int64_t u) {
        const int64_t y1 = 2 * u, y2 = 2 * u + 1;
        const bool l1 = y1 < io.nsys, l2 = y2 < io.nsys;
        const double* x1 = io.in + io.in_off + (l1 ? y1 : 0) * io.in_stride;
        const double* x2 = io.in + io.in_off + (l2 ? y2 : 0) * io.in_stride;
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            p1[i] = l1 ? x1[j + i * TPS] : 0.0;
            p2[i] = l2 ? x2[j + i * TPS] : 0.0;
        }
    };
    int64_t u = (int64_t)blockIdx.x * S::SPC + s;
    fetch(u);
    for (int64_t base = (int64_t)blockIdx.x * S::SPC; base < npairs; base += stride_units, u += stride_units) {
        if constexpr (TYPE == 2) {
            // natural order; the first stage reads it in Makhoul's
#pragma unroll
            for (int i = 0; i < PER; ++i) buf[dct_pad(j + i * TPS)] = make_double2(p1[i], p2[i]);
        } else {
            // unpadded here, so that the descending reads of X_{N-k} touch 8
            // different bank groups per access phase
#pragma unroll
            for (int i = 0; i < PER; ++i) buf[j + i * TPS] = make_double2(p1[i], p2[i]);
            sync();
            double2 Xr[PER];
#pragma unroll
            for (int i = 0; i < PER; ++i) {
                const int k = j + i * TPS;
                Xr[i] = (k == 0) ? make_double2(0.0, 0.0) : buf[N - k];
            }
            sync();
#pragma unroll
            for (int i = 0; i < PER; ++i) {
                const int k = j + i * TPS;
                const double2 c = __ldg(&pt[k]);
                // z_k = e^{-i t} (X_k + i X_{N-k}) = (X_k cos t + X_{N-k} sin t) + i (X_{N-k} cos t - X_k sin t)
                const double z1r = __fma_rn(p1[i], c.x, Xr[i].x * c.y), z1i = __fma_rn(Xr[i].x, c.x, -(p1[i] * c.y));
                const double z2r = __fma_rn(p2[i], c.x, Xr[i].y * c.y), z2i = __fma_rn(Xr[i].y, c.x, -(p2[i] * c.y));
                buf[dct_pad(k)] = make_double2(z1r - z2i, z1i + z2r);  // z1 + i z2
            }
        }
        sync();
        fetch(u + stride_units);  // in flight while this pair is transformed
        // The stages: the first reads type 2's rows in Makhoul's order, the
        // last writes type 3's results in the rows' order and type 2's
        // without the pads.
        constexpr int LAST = TYPE == 3 ? 1 : 2;
        constexpr int OUT8 = S::REM == 0 ? LAST : 0;  // the last radix-8 stage is the last
        dct_stage<8, N, TPS, TYPE == 2, S::L8 == 1 ? OUT8 : 0>(buf, 1, j, tws, sync);
        int Ns = 8;
#pragma unroll 1
        for (int st = 1; st < S::L8 - 1; ++st) {
            dct_stage<8, N, TPS>(buf, Ns, j, tws, sync);
            Ns *= 8;
        }
        if constexpr (S::L8 >= 2) {
            dct_stage<8, N, TPS, false, OUT8>(buf, Ns, j, tws, sync);
            Ns *= 8;
        }
        if constexpr (S::REM == 1) dct_stage<2, N, TPS, false, LAST>(buf, Ns, j, tws, sync);
        else if constexpr (S::REM == 2) dct_stage<4, N, TPS, false, LAST>(buf, Ns, j, tws, sync);
        const int64_t y1 = 2 * u, y2 = 2 * u + 1;
        const bool l1 = y1 < io.nsys, l2 = y2 < io.nsys;
        double* o1 = io.out + io.out_off + (l1 ? y1 : 0) * io.out_stride;
        double* o2 = io.out + io.out_off + (l2 ? y2 : 0) * io.out_stride;
        if constexpr (TYPE == 2) {
#pragma unroll
            for (int i = 0; i < PER; ++i) {
                const int k = j + i * TPS;
                const double2 Z = buf[k], Zr = buf[(N - k) & (N - 1)];  // unpadded (the last stage)
                const double2 c = __ldg(&pt[k]);
                if (l1) o1[k] = __fma_rn(Z.x + Zr.x, c.x, (Z.y - Zr.y) * c.y);
                if (l2) o2[k] = __fma_rn(Z.y + Zr.y, c.x, -((Z.x - Zr.x) * c.y));
            }
        } else {
#pragma unroll
            for (int i = 0; i < PER; ++i) {
                const double2 Z = buf[dct_pad(j + i * TPS)];  // in the rows' order (the last stage)
                if (l1) o1[j + i * TPS] = Z.x;
                if (l2) o2[j + i * TPS] = Z.y;
            }
        }
        sync();  // the buffer takes the next round's pair
    }
}

}  // namespace pfb
