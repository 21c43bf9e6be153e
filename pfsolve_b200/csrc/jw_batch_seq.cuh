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
// Data movement, per chunk of CH = 8 or 16 rows x 32 systems:
//  * In: a real box and an imaginary box of CH rows x 32 systems (64-byte
//    swizzle for 8 rows, 128-byte for 16).  The entry's input is one 2-D tensor of nsys rows of
//    2*in_stride doubles (a system's real rows, then its imaginary rows), so
//    both boxes are TMA loads from one map; the imaginary box starts at
//    in_stride + r0.  With an odd stride that start is 8 bytes off a 16-byte
//    boundary, so the box is taken one row higher (descending sweep: rows
//    r0+1 .. r0+CH) or lower (ascending: r0-1 .. r0+CH-2); the one row outside
//    comes from the next chunk's box, and for the last chunk from an extra
//    imaginary-only chunk (sweep index Q).  Rows at or beyond M that the boxes
//    still cover (the imaginary rows after the real ones, stride padding) are
//    zeroed in registers.  Inputs that are not 16-byte aligned take 8-byte
//    cp.async copies into the same layout instead.
//  * Coefficients: a pre-pass kernel (one CTA per entry) forms every row's
//    {w_{-1}, w_0, w_{+1}, solve band, Scale factor} once per launch -- the
//    bands are read at launch time, as the reference does -- into a table of
//    48-byte rows; a chunk's CH rows come with its boxes as one
//    bulk copy, into a ring of NBUF + 1 slots (one more than the data buffers,
//    so a refill never lands on the rows being read), read by broadcast.
//  * Completion: one mbarrier per data buffer; lane 0 posts the transaction
//    bytes, every lane arrives once per chunk (through
//    cp.async.mbarrier.arrive.noinc on the cp.async path).  Waits are bounded:
//    one that runs out records kStatusWaitTimeout and the warp stops.
//  * Out: a lane reads its rows into registers, the buffer is refilled at
//    once, the rows are computed in registers, 8 at a time, and written
//    packed into a staging buffer (128-byte swizzle, boxes of 8 rows) that
//    one TMA store per 8 rows writes back; the output map's rows end at 2*M, so padding is never written.
#pragma once
#include <cuda.h>

#include "jw_steps_seq.cuh"
#include "jw_variants.h"

namespace pfb {

// A chunk holds CH rows (8 or 16) of 32 systems: a real and an imaginary box
// of CH doubles per system (64-byte swizzle for 8 rows, 128-byte for 16), a
// staging buffer of CH packed rows per system (128-byte swizzle, in boxes of 8
// rows), and CH coefficient rows.
constexpr int kBsCoefRowBytes = 48;  // w_{-1}, w_0, w_{+1}, band, Scale, 0
template <int CH>
struct BsGeom {
    static constexpr int BOX = 32 * CH * 8;     // one box: CH doubles x 32 systems
    static constexpr int IN = 2 * BOX;          // real box | imaginary box
    static constexpr int OUT = 32 * CH * 16;    // CH packed rows x 32 systems
    static constexpr int COEF = CH * kBsCoefRowBytes;
    static constexpr int UNITS = CH / 2;        // 16-byte units per system row of a box
};

// Per warp: NBUF input buffers and one staging buffer (after a 1024-byte
// aligned base), and elsewhere NBUF + 1 coefficient slots and NBUF mbarriers.
__host__ __device__ constexpr size_t batch_seq_buf_bytes(int CH, int NBUF)
{
    return (size_t)NBUF * 2 * 32 * CH * 8 + (size_t)32 * CH * 16;
}
__host__ __device__ constexpr size_t batch_seq_aux_bytes(int CH, int NBUF)
{
    return ((size_t)(NBUF + 1) * CH * kBsCoefRowBytes + (size_t)NBUF * 8 + 127) / 128 * 128;  // 16-byte aligned slots
}
__host__ __device__ constexpr size_t batch_seq_smem_bytes(int CH, int NBUF, int NW)
{
    return 1024 + (size_t)NW * (batch_seq_buf_bytes(CH, NBUF) + batch_seq_aux_bytes(CH, NBUF));
}
// Coefficient rows of an entry of M rows: padded to whole chunks of 16 rows.
__host__ __device__ constexpr int64_t batch_seq_coef_rows(int64_t M) { return (M + 15) & ~int64_t(15); }

__device__ __forceinline__ void cp_async8_n(uint32_t dst, const void* src, int bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_mbar_arrive(uint32_t bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Pre-pass: coefficient rows of entry blockIdx.x (zeros at and beyond M).
template <int SVK>
__global__ void __launch_bounds__(128) jw_batch_seq_coef_kernel(const BatchEntryDev* __restrict__ entries,
                                                                const BatchSeqEntry* __restrict__ seq,
                                                                double* __restrict__ coefs)
{
    const int e = blockIdx.x;
    const JwOperator op = entries[e].op;
    const int M = (int)op.M;
    const int rows = (int)batch_seq_coef_rows(M);
    double2* t = reinterpret_cast<double2*>(coefs + 6 * seq[e].coef_off);
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

// Per-warp pipeline state kept across work items: chunks of earlier items
// (chunk c of the warp's lifetime uses buffer c % NBUF and coefficient slot
// c % (NBUF + 1)) and the parity of every buffer's next completion.
struct BsPipe {
    uint32_t base;
    uint32_t phases;
};

// Byte offset of 16-byte unit u of system row s in a box of CH doubles per
// row (the TMA swizzle of that box: 64-byte rows for 8, 128-byte for 16).
template <int CH>
__device__ __forceinline__ uint32_t bs_unit_off(int s, int u)
{
    if constexpr (CH == 8) return s * 64 + ((u ^ ((s >> 1) & 3)) << 4);
    else return s * 128 + ((u ^ (s & 7)) << 4);
}

// Sweep of one work item: systems y0 .. y0+ns-1 of entry `ent`, chunks of CH
// rows.  LAY: 0 TMA with an even stride, 1 TMA with an odd stride (shifted
// imaginary box), 2 8-byte cp.async copies.  Returns false when a wait ran out.
template <int SVK, int CH, int NBUF, int LAY>
__device__ __forceinline__ bool batch_seq_item(const BatchEntryDev* __restrict__ ent,
                                               const BatchSeqEntry* __restrict__ sq, const double* __restrict__ ctab,
                                               int64_t y0, int ns, uint32_t bufs_u, uint32_t aux_u, int lane,
                                               BsPipe& pipe)
{
    using G = BsGeom<CH>;
    constexpr int NU = G::UNITS;
    constexpr bool DESC = (SVK == SV_UPPER);
    constexpr bool SHIFT = (LAY == 1);
    const CUtensorMap* imap = &sq->in[CH == 16 ? 1 : 0];
    const int M = (int)ent->io.M;
    const int istr = (int)ent->io.in_stride;
    const double scaleC = ent->op.scaleC;
    const int Q = (M + CH - 1) / CH;
    const int nch = SHIFT ? Q + 1 : Q;  // chunks of this item (SHIFT: and the imaginary-only one)
    const int y0i = (int)y0;
    const double* in0 = ent->io.in + ent->io.in_off;
    const double* re0 = in0 + 2 * y0 * ent->io.in_stride;
    const uint32_t bars_u = aux_u + (NBUF + 1) * G::COEF;
    const uint32_t stage_u = bufs_u + NBUF * G::IN;
    const int swo = lane & 7;  // 128-byte swizzle of this lane's staging row

    auto slot = [&](int c) -> uint32_t { return (pipe.base + (uint32_t)c) % NBUF; };
    auto buf_of = [&](int c) -> uint32_t { return bufs_u + slot(c) * G::IN; };
    auto coef_of = [&](int c) -> uint32_t { return aux_u + ((pipe.base + (uint32_t)c) % (NBUF + 1)) * G::COEF; };
    // chunk c: boxes and coefficient rows, one arrival per lane
    auto issue = [&](int c) {
        if (c >= nch) return;
        const int r0 = CH * (DESC ? Q - 1 - c : c);  // SHIFT's extra chunk: q = -1 or Q
        const bool rows_chunk = c < Q;
        const uint32_t buf = buf_of(c), bar = bars_u + slot(c) * 8;
        if constexpr (LAY != 2) {
            if (lane == 0) {
                const int xi = istr + r0 + (SHIFT ? (DESC ? 1 : -1) : 0);
                mbar_expect_tx(bar, rows_chunk ? G::IN + G::COEF : G::BOX);
                if (rows_chunk) {
                    tma_load_2d(buf, imap, r0, y0i, bar);
                    bulk_load(coef_of(c), ctab + 6 * r0, G::COEF, bar);
                }
                tma_load_2d(buf + G::BOX, imap, xi, y0i, bar);
            }
            __syncwarp();
            mbar_arrive(bar);
        } else {
            if (lane == 0) {
                mbar_expect_tx(bar, G::COEF);
                bulk_load(coef_of(c), ctab + 6 * r0, G::COEF, bar);
            }
            __syncwarp();
            // piece p = lane + 32 t: system p / (2 CH), part (p / CH) % 2, row p % CH
            constexpr int SPT = 16 / CH;  // systems per 32 pieces
#pragma unroll
            for (int t = 0; t < 2 * CH; ++t) {
                const int p = lane + 32 * t;
                const int s = p / (2 * CH), part = (p / CH) & 1, rr = p % CH;
                const int row = r0 + rr;
                const bool ok = s < ns && row < M;
                const double* src = re0 + (int64_t)(2 * s + part) * ent->io.in_stride + row;
                cp_async8_n(buf + part * G::BOX + bs_unit_off<CH>(s, rr >> 1) + ((rr & 1) << 3), ok ? src : in0,
                            ok ? 8 : 0);
                (void)SPT;
            }
            cp_async_mbar_arrive(bar);
        }
    };
    // wait for chunk c; false when the wait ran out
    auto wait = [&](int c) -> bool {
        const uint32_t b = slot(c);
        const bool w = __all_sync(FULL, mbar_wait_bounded(bars_u + b * 8, (pipe.phases >> b) & 1u));
        if (w) pipe.phases ^= 1u << b;
        return w;
    };
    // after a timeout: give the chunks issued in [c0, c1) a bounded wait each,
    // so that no copy is left landing in shared memory
    auto drain = [&](int c0, int c1) {
        for (int c = c0; c < c1 && c < nch; ++c) (void)mbar_wait_bounded(bars_u + slot(c) * 8, (pipe.phases >> slot(c)) & 1u);
    };
    auto lds2 = [](uint32_t a) -> double2 {
        double2 v;
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "r"(a));
        return v;
    };
    // 16-byte unit u of this lane's row of a box
    auto unit = [&](uint32_t box, int u) { return lds2(box + bs_unit_off<CH>(lane, u)); };

#pragma unroll
    for (int c = 0; c < NBUF; ++c) issue(c);
    if (!wait(0)) {
        drain(0, NBUF);
        return false;
    }

    double cr = 0.0, ci = 0.0;  // right-hand side of the previous sweep row
    double zr = 0.0, zi = 0.0;  // solution of the previous sweep row
    for (int k = 0; k < Q; ++k) {
        const int r0 = CH * (DESC ? Q - 1 - k : k);
        if (k + 1 < nch && !wait(k + 1)) {
            drain(k + 1, k + NBUF);
            return false;
        }
        const uint32_t cb = buf_of(k), nb = buf_of(k + 1);
        double br[CH], bi[CH];
#pragma unroll
        for (int u = 0; u < NU; ++u) {
            const double2 vr = unit(cb, u);
            br[2 * u] = vr.x;
            br[2 * u + 1] = vr.y;
        }
        // first sweep row of the next chunk (row r0 - 1 descending, r0 + CH ascending)
        double lr = 0.0, li = 0.0;
        if constexpr (SHIFT) {
            // imaginary box: rows r0+1 .. r0+CH (descending) or r0-1 .. r0+CH-2 (ascending)
#pragma unroll
            for (int u = 0; u < NU; ++u) {
                const double2 vi = unit(cb + G::BOX, u);
                if constexpr (DESC) {
                    bi[2 * u + 1] = vi.x;
                    if (u < NU - 1) bi[2 * u + 2] = vi.y;
                } else {
                    if (u > 0) bi[2 * u - 1] = vi.x;
                    bi[2 * u] = vi.y;
                }
            }
            const double2 n = unit(nb + G::BOX, DESC ? NU - 1 : 0);  // rows r0-1, r0 / r0+CH-1, r0+CH
            if constexpr (DESC) {
                bi[0] = n.y;
                if (k + 1 < Q) li = n.x;
            } else {
                bi[CH - 1] = n.x;
                li = n.y;
            }
        } else {
#pragma unroll
            for (int u = 0; u < NU; ++u) {
                const double2 vi = unit(cb + G::BOX, u);
                bi[2 * u] = vi.x;
                bi[2 * u + 1] = vi.y;
            }
            if (k + 1 < Q) li = DESC ? unit(nb + G::BOX, NU - 1).y : unit(nb + G::BOX, 0).x;
        }
        if (k + 1 < Q) lr = DESC ? unit(nb, NU - 1).y : unit(nb, 0).x;
        // rows at or beyond M that the boxes cover are not data
        if (r0 + CH > M) {
#pragma unroll
            for (int j = 0; j < CH; ++j)
                if (r0 + j >= M) {
                    br[j] = 0.0;
                    bi[j] = 0.0;
                }
        }
        if (!DESC && r0 + CH >= M) {
            lr = 0.0;
            li = 0.0;
        }
        const uint32_t tab = coef_of(k);
        __syncwarp();  // every lane holds its rows: the buffer takes chunk k + NBUF
        issue(k + NBUF);
        // the staging buffer is free once the previous chunk's stores have read it
        if (lane == 0) bulk_wait_read_all();
        __syncwarp();
        // rows in sweep order, 8 at a time: results stay in registers until
        // the group's staging stores, so the coefficient loads run ahead
#pragma unroll
        for (int h = 0; h < CH / 8; ++h) {
            double2 res[8];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
                const int ss = 8 * h + jj;               // sweep step within the chunk
                const int j = DESC ? CH - 1 - ss : ss;   // row r0 + j
                const int jn = DESC ? j - 1 : j + 1;     // next sweep row inside the chunk
                const double nr = (ss < CH - 1) ? br[jn] : lr, ni = (ss < CH - 1) ? bi[jn] : li;
                const double mr = DESC ? nr : cr, mi = DESC ? ni : ci;  // row i - 1
                const double pr = DESC ? cr : nr, pi = DESC ? ci : ni;  // row i + 1
                const double2 w01 = lds2(tab + kBsCoefRowBytes * j);
                const double2 w2c = lds2(tab + kBsCoefRowBytes * j + 16);
                const double2 scz = lds2(tab + kBsCoefRowBytes * j + 32);
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
                res[jj] = make_double2(scz.x * orr, scz.x * oii);
                cr = br[j];
                ci = bi[j];
            }
#pragma unroll
            for (int jj = 0; jj < 8; ++jj) {
                const int j = DESC ? CH - 1 - (8 * h + jj) : 8 * h + jj;
                const uint32_t a = stage_u + (j >> 3) * (32 * 128) + lane * 128 + (((j & 7) ^ swo) << 4);
                asm volatile("st.shared.v2.f64 [%0], {%1, %2};\n" ::"r"(a), "d"(res[jj].x), "d"(res[jj].y) : "memory");
            }
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
#pragma unroll
            for (int h = 0; h < CH / 8; ++h) tma_store_2d(&sq->out, 2 * (r0 + 8 * h), y0i, stage_u + h * (32 * 128));
            bulk_commit();
        }
    }
    pipe.base += (uint32_t)nch;
    return true;
}

// NW warps per CTA, each a consumer of the batch's work queue.
template <int SVK, int CH, int NBUF, int NW>
__global__ void __launch_bounds__(32 * NW, 1) jw_batch_seq_kernel(const BatchEntryDev* __restrict__ entries,
                                                                const BatchSeqEntry* __restrict__ seq,
                                                                const double* __restrict__ coefs,
                                                                const WorkItem* __restrict__ items,
                                                                const int nitems, unsigned int* __restrict__ counter)
{
    static_assert(NBUF >= 3, "the lookahead chunk and one more must be in flight");
    static_assert(CH == 8 || CH == 16, "chunk rows");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t raw_u = smem_u32(smem_raw);
    const uint32_t base_u = raw_u + ((1024u - (raw_u & 1023u)) & 1023u);
    const uint32_t bufs_u = base_u + warp * (uint32_t)batch_seq_buf_bytes(CH, NBUF);
    const uint32_t aux_u =
        base_u + NW * (uint32_t)batch_seq_buf_bytes(CH, NBUF) + warp * (uint32_t)batch_seq_aux_bytes(CH, NBUF);
    if (lane < NBUF) mbar_init(aux_u + (NBUF + 1) * BsGeom<CH>::COEF + 8 * lane, 32);
    mbar_init_fence();
    __syncwarp();
    BsPipe pipe{0u, 0u};
    for (;;) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(counter, 1u);
        it = __shfl_sync(FULL, it, 0);
        if (it >= nitems) break;
        const WorkItem wi = items[it];
        const BatchEntryDev* ent = entries + wi.entry;
        const BatchSeqEntry* sq = seq + wi.entry;
        const double* ctab = coefs + 6 * sq->coef_off;
        const int ns = (int)(wi.y1 - wi.y0);
        bool ok;
        if (!sq->tma_in) ok = batch_seq_item<SVK, CH, NBUF, 2>(ent, sq, ctab, wi.y0, ns, bufs_u, aux_u, lane, pipe);
        else if (ent->io.in_stride & 1)
            ok = batch_seq_item<SVK, CH, NBUF, 1>(ent, sq, ctab, wi.y0, ns, bufs_u, aux_u, lane, pipe);
        else ok = batch_seq_item<SVK, CH, NBUF, 0>(ent, sq, ctab, wi.y0, ns, bufs_u, aux_u, lane, pipe);
        if (!ok) {
            if (lane == 0) atomicOr(&g_stream_status, kStatusWaitTimeout);
            break;
        }
    }
    if (lane == 0) bulk_wait_all();
}

}  // namespace pfb
