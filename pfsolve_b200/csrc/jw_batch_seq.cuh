// jw_batch_seq.cuh -- uneven batches of bidiagonal JW steps with one complex
// system per lane, every system's rows in one sweep.
//
// Operators whose effective matvec V*A couples rows i-1, i, i+1 and whose
// solve has a unit diagonal and one off-diagonal band
// (pfSolve_KernelsLevel2/pfSolve_JonesWorland.h:108-374):
//
//   SV_UPPER (rows descending):  z_i = y_i - h_i z_{i+1}
//   SV_LOWER (rows ascending):   z_i = y_i - l_i z_{i-1}
//   SV_NONE  (rows ascending):   z_i = y_i
//
// with y = V*A*b, XXII input (a system's real rows, then its imaginary rows),
// packed complex output and the fused Scale epilogue of the block kernel
// (pfSolve_ReadWrite.h:2293-2354, pfSolve_RegistersScaleC.h:27-201).  Solution
// row 0 is multiplied by scaleC after the solve, as in the group kernel.
//
// A warp takes work items of up to 32 systems of one entry from the batch's
// queue.  Lane s owns system y0 + s and walks its rows in sweep order,
// carrying the recurrence (and the previous right-hand side row) in registers:
// no scans and no cross-lane traffic, the real and imaginary chains give two
// independent FP64 dependency chains per lane.
//
// Staging: chunks of 8 rows x 32 systems (4 KB).  A system's slot is 128 bytes
// -- units 0..3 hold real rows (0,1) .. (6,7), units 4..7 the imaginary rows --
// with 16-byte unit u stored at u ^ (s & 7), so that a lane's reads of its own
// slot and the warp's coalesced copies (8 lanes per system) hit distinct bank
// groups.  cp.async keeps NBUF chunks in flight per warp; bytes beyond the
// system's M rows are zero-filled.  Three copy layouts:
//   BS_ALIGNED  input 16-byte aligned, even stride: 16-byte copies.
//   BS_SHIFTED  input 16-byte aligned, odd stride (odd M, packed): the real
//               rows are 16-byte aligned, the imaginary rows 8 bytes off, so
//               a chunk's imaginary units hold rows r0+1 .. r0+8 (descending
//               sweep) or r0-1 .. r0+6 (ascending) -- still 16-byte copies.
//               The one row outside comes from the next chunk's buffer; for
//               the last chunk an extra one-unit chunk (sweep index Q) holds
//               it.  The row the shifted units read at -1 lies inside the
//               system's real rows and is never used.
//   BS_UNALIGNED anything else: 8-byte copies.  Row i needs the next sweep row's right-hand side,
// so the chunk after the current one has landed before a chunk is processed.
// A lane reads its slot into registers, computes its 8 rows in registers
// (no shared-memory stores inside the row loop, so the coefficient loads run
// ahead), then writes the packed results into its slot; the warp leaves them
// as coalesced 16-byte streaming stores and refills the buffer.
//
// Coefficients: a pre-pass kernel (one CTA per entry) forms every row's
// {w_{-1}, w_0, w_{+1}, solve band, Scale factor} once per launch -- the bands
// are read at launch time, as the reference does -- into a table of 48-byte
// rows; each chunk's 8 table rows (384 bytes) travel in the chunk's cp.async
// group into a ring of NBUF + 1 slots (one more than the data buffers, so a
// refill never lands on the rows being read) and are read by broadcast.
#pragma once
#include "jw_kernel.cuh"

namespace pfb {

constexpr int kBsDataBytes = 32 * 128;  // 32 systems x 8 units of 16 bytes
constexpr int kBsCoefRowBytes = 48;     // w_{-1}, w_0, w_{+1}, band, Scale, 0
constexpr int kBsCoefBytes = 8 * kBsCoefRowBytes;

__host__ __device__ constexpr size_t batch_seq_warp_bytes(int NBUF)
{
    return (size_t)NBUF * kBsDataBytes + (size_t)(NBUF + 1) * kBsCoefBytes;
}
__host__ __device__ constexpr size_t batch_seq_smem_bytes(int NBUF, int NW) { return NW * batch_seq_warp_bytes(NBUF); }
// Coefficient rows of an entry of M rows: padded to whole chunks.
__host__ __device__ constexpr int64_t batch_seq_coef_rows(int64_t M) { return (M + 7) & ~int64_t(7); }

__device__ __forceinline__ void cp_async16_n(uint32_t dst, const void* src, int bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async8_n(uint32_t dst, const void* src, int bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

// Pre-pass: coefficient rows of entry blockIdx.x at coefs + 6 coef_off[e]
// (zeros at and beyond M).
template <int SVK>
__global__ void __launch_bounds__(128) jw_batch_seq_coef_kernel(const BatchEntryDev* __restrict__ entries,
                                                                const int64_t* __restrict__ coef_off,
                                                                double* __restrict__ coefs)
{
    const int e = blockIdx.x;
    const JwOperator op = entries[e].op;
    const int M = (int)op.M;
    const int rows = (int)batch_seq_coef_rows(M);
    double2* t = reinterpret_cast<double2*>(coefs + 6 * coef_off[e]);
    for (int i = threadIdx.x; i < rows; i += blockDim.x) {
        double w[3] = {0.0, 0.0, 0.0};
        double c = 0.0, sc = 0.0;
        if (i < M) {
            jw_row_weights<1, 3>(op, i, w);
            if constexpr (SVK == SV_UPPER) c = (i < M - 1) ? band(op, op.off_su, i) : 0.0;
            if constexpr (SVK == SV_LOWER) c = (i >= 1) ? band(op, op.off_sl, i) : 0.0;
            sc = op.scale_kind ? scale_factor(op.scale_kind, i, op.lshift, op.scale_s) : 1.0;
        }
        t[3 * i] = make_double2(w[0], w[1]);
        t[3 * i + 1] = make_double2(w[2], c);
        t[3 * i + 2] = make_double2(sc, 0.0);
    }
}

enum : int { BS_ALIGNED = 0, BS_SHIFTED = 1, BS_UNALIGNED = 2 };

// Sweep of one work item: systems y0 .. y0+ns-1 of entry `ent`, coefficient
// rows at `ctab`, copy layout LAY.
template <int SVK, int NBUF, int LAY>
__device__ __forceinline__ void batch_seq_item(const BatchEntryDev* __restrict__ ent, const double* __restrict__ ctab,
                                               int64_t y0, int ns, unsigned char* wbase, int lane)
{
    constexpr bool DESC = (SVK == SV_UPPER);
    const uint32_t wbase_u = static_cast<uint32_t>(__cvta_generic_to_shared(wbase));
    const int sw = lane & 7;   // swizzle of this lane's own slot
    const int pu = lane & 7;   // unit of the coalesced copies
    const int ps = lane >> 3;  // system within each group of 4 of the coalesced copies
    const int M = (int)ent->io.M;
    const int64_t istr = ent->io.in_stride, ostr = ent->io.out_stride;
    const double* in0 = ent->io.in + ent->io.in_off;
    const double* re0 = in0 + 2 * y0 * istr;  // real rows of system y0
    double2* out0 = reinterpret_cast<double2*>(ent->io.out) + ent->io.out_off + y0 * ostr;
    const double scaleC = ent->op.scaleC;
    const int Q = (M + 7) >> 3;

    // chunk of sweep index k: data into buffer k % NBUF, coefficient rows into
    // slot k % (NBUF + 1); an empty group past the end (BS_SHIFTED: sweep index
    // Q is the one-unit chunk of the row beyond the last chunk)
    constexpr int kVirtUnit = DESC ? 7 : 4;  // BS_SHIFTED: the unit of sweep index Q
    auto issue = [&](int k) {
        if (k < Q || (LAY == BS_SHIFTED && k == Q)) {
            const int r0 = 8 * (DESC ? Q - 1 - k : k);
            const uint32_t dst0 = wbase_u + (uint32_t)((k % NBUF) * kBsDataBytes);
            if (lane < 24 && k < Q)
                cp_async16_n(wbase_u + NBUF * kBsDataBytes + (k % (NBUF + 1)) * kBsCoefBytes + 16 * lane,
                             ctab + 6 * r0 + 2 * lane, 16);
            if constexpr (LAY != BS_UNALIGNED) {
                // imaginary units of BS_SHIFTED start one row up (descending) or down
                const int shift = (LAY == BS_SHIFTED && pu >= 4) ? (DESC ? 1 : -1) : 0;
                const int row = r0 + 2 * (pu & 3) + shift;
                const int nb = (M - row >= 2) ? 16 : (M - row == 1 ? 8 : 0);
                const double* src = re0 + (int64_t)(2 * ps + (pu >> 2)) * istr + row;
                const bool want = k < Q || pu == kVirtUnit;
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const int s = 4 * t + ps;
                    const int bytes = (s < ns) ? nb : 0;
                    if (want)
                        cp_async16_n(dst0 + s * 128 + ((pu ^ (s & 7)) << 4),
                                     bytes ? src + (int64_t)(8 * t) * istr : in0, bytes);
                }
            } else {
                const int part = (lane >> 3) & 1, rr = lane & 7;
                const int row = r0 + rr;
                const int u = part * 4 + (rr >> 1);
                const double* src = re0 + (int64_t)(2 * (lane >> 4) + part) * istr + row;
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    // piece lane + 32 t: system 2 t + lane / 16, part (lane / 8) % 2, row lane % 8
                    const int s = 2 * t + (lane >> 4);
                    const bool ok = s < ns && row < M;
                    cp_async8_n(dst0 + s * 128 + ((u ^ (s & 7)) << 4) + ((rr & 1) << 3),
                                ok ? src + (int64_t)(4 * t) * istr : in0, ok ? 8 : 0);
                }
            }
        }
        cp_async_commit();
    };

#pragma unroll
    for (int k = 0; k < NBUF; ++k) issue(k);

    double cr = 0.0, ci = 0.0;  // right-hand side of the previous sweep row
    double zr = 0.0, zi = 0.0;  // solution of the previous sweep row
    for (int k = 0; k < Q; ++k) {
        const int q = DESC ? Q - 1 - k : k;
        const int r0 = 8 * q;
        cp_async_wait<NBUF - 2>();
        __syncwarp();
        const unsigned char* cb = wbase + (k % NBUF) * kBsDataBytes + lane * 128;
        const double* tab =
            reinterpret_cast<const double*>(wbase + NBUF * kBsDataBytes + (k % (NBUF + 1)) * kBsCoefBytes);
        const unsigned char* nb = wbase + ((k + 1) % NBUF) * kBsDataBytes + lane * 128;  // next chunk's slot
        auto unit = [&](const unsigned char* b, int u) { return *reinterpret_cast<const double2*>(b + ((u ^ sw) << 4)); };
        double br[8], bi[8];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double2 vr = unit(cb, u);
            br[2 * u] = vr.x;
            br[2 * u + 1] = vr.y;
        }
        // first sweep row of the next chunk (row r0 - 1 descending, r0 + 8 ascending)
        double lr = 0.0, li = 0.0;
        if constexpr (LAY == BS_SHIFTED) {
            // imaginary units: rows r0+1 .. r0+8 (descending) or r0-1 .. r0+6 (ascending)
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const double2 vi = unit(cb, u + 4);
                if constexpr (DESC) {
                    bi[2 * u + 1] = vi.x;
                    if (u < 3) bi[2 * u + 2] = vi.y;
                } else {
                    if (u > 0) bi[2 * u - 1] = vi.x;
                    bi[2 * u] = vi.y;
                }
            }
            const double2 n = unit(nb, kVirtUnit);  // rows r0-1, r0 (descending) or r0+7, r0+8
            if constexpr (DESC) {
                bi[0] = n.y;
                if (k + 1 < Q) li = n.x;
            } else {
                bi[7] = n.x;
                li = n.y;
            }
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const double2 vi = unit(cb, u + 4);
                bi[2 * u] = vi.x;
                bi[2 * u + 1] = vi.y;
            }
            if (k + 1 < Q) li = DESC ? unit(nb, 7).y : unit(nb, 4).x;
        }
        if (k + 1 < Q) lr = DESC ? unit(nb, 3).y : unit(nb, 0).x;
        double2 res[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
            const int j = DESC ? 7 - jj : jj;
            // rows i-1 and i+1 of row i = r0 + j
            const int jn = DESC ? j - 1 : j + 1;  // next sweep row inside the chunk
            const double nr = (jj < 7) ? br[jn] : lr, ni = (jj < 7) ? bi[jn] : li;
            const double mr = DESC ? nr : cr, mi = DESC ? ni : ci;
            const double pr = DESC ? cr : nr, pi = DESC ? ci : ni;
            const double* t = tab + 6 * j;
            const double2 w01 = *reinterpret_cast<const double2*>(t);
            const double2 w2c = *reinterpret_cast<const double2*>(t + 2);
            const double sc = t[4];
            double yr = w01.x * mr, yi = w01.x * mi;
            yr = __fma_rn(w01.y, br[j], yr);
            yi = __fma_rn(w01.y, bi[j], yi);
            yr = __fma_rn(w2c.x, pr, yr);
            yi = __fma_rn(w2c.x, pi, yi);
            if constexpr (SVK != SV_NONE) {
                zr = __fma_rn(-w2c.y, zr, yr);
                zi = __fma_rn(-w2c.y, zi, yi);
            } else {
                zr = yr;
                zi = yi;
            }
            double orr = zr, oii = zi;
            if (SVK != SV_NONE && r0 + j == 0) {
                orr = scaleC * orr;
                oii = scaleC * oii;
            }
            res[j] = make_double2(sc * orr, sc * oii);
            cr = br[j];
            ci = bi[j];
        }
        unsigned char* ob = wbase + (k % NBUF) * kBsDataBytes;
        __syncwarp();  // every lane has read its slot and lookahead row
#pragma unroll
        for (int j = 0; j < 8; ++j) *reinterpret_cast<double2*>(ob + lane * 128 + ((j ^ sw) << 4)) = res[j];
        __syncwarp();
        const int row = r0 + pu;
        double2* dst = out0 + (int64_t)ps * ostr + row;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int s = 4 * t + ps;
            const double2 v = *reinterpret_cast<const double2*>(ob + s * 128 + ((pu ^ (s & 7)) << 4));
            if (s < ns && row < M) __stcs(dst + (int64_t)(4 * t) * ostr, v);
        }
        __syncwarp();
        issue(k + NBUF);
    }
}

// NW warps per CTA, each a consumer of the batch's work queue.
template <int SVK, int NBUF, int NW>
__global__ void __launch_bounds__(32 * NW, 1) jw_batch_seq_kernel(const BatchEntryDev* __restrict__ entries,
                                                                const int64_t* __restrict__ coef_off,
                                                                const double* __restrict__ coefs,
                                                                const WorkItem* __restrict__ items,
                                                                const int nitems, unsigned int* __restrict__ counter)
{
    static_assert(NBUF >= 3, "the lookahead chunk and one more must be in flight");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* wbase = smem_raw + (size_t)warp * batch_seq_warp_bytes(NBUF);
    for (;;) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(counter, 1u);
        it = __shfl_sync(FULL, it, 0);
        if (it >= nitems) break;
        const WorkItem wi = items[it];
        const BatchEntryDev* ent = entries + wi.entry;
        const double* ctab = coefs + 6 * coef_off[wi.entry];
        const bool al16 = (reinterpret_cast<uintptr_t>(ent->io.in + ent->io.in_off) & 15) == 0;
        const int ns = (int)(wi.y1 - wi.y0);
        if (al16 && (ent->io.in_stride & 1) == 0) batch_seq_item<SVK, NBUF, BS_ALIGNED>(ent, ctab, wi.y0, ns, wbase, lane);
        else if (al16) batch_seq_item<SVK, NBUF, BS_SHIFTED>(ent, ctab, wi.y0, ns, wbase, lane);
        else batch_seq_item<SVK, NBUF, BS_UNALIGNED>(ent, ctab, wi.y0, ns, wbase, lane);
    }
    cp_async_wait<0>();
}

}  // namespace pfb
