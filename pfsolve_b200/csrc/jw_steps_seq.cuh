// jw_steps_seq.cuh -- K consecutive bidiagonal JW steps, one system per lane,
// all K steps pipelined in one sweep over the rows.
//
// Operator of upperBanded 1 / 0 with jw_type % 10 in {0, 1, 2} and K > 1
// (pfSolve_KernelsLevel2/pfSolve_JonesWorland.h:108-374; semantics as in
// jw_steps.cuh).  For these kinds every step is one directional recurrence:
//
//   upperBanded 1 (rows ascending):  y_i = d_i x_i + u_i x_{i+1},  z_i = y_i - l_i z_{i-1}
//   upperBanded 0 (rows descending): y_i = d_i x_i + l_i x_{i-1},  z_i = y_i - u_i z_{i+1}
//
// so step s at row i needs step s-1 only at rows i and i+1 (in sweep order).
// A lane therefore runs step s one row behind step s-1: at each sweep
// position it advances all K steps by one row, holding two values per step in
// registers.  The data crosses HBM once, there is no cross-lane communication
// and no barrier; the per-row coefficients are read from a shared table by
// all lanes at the same address (broadcast).
//
// Staging: a warp owns 32 consecutive systems; their rows move in boxes of
// CH = 8 or 16 rows x 32 systems (2 or 4 KB; 64- or 128-byte swizzle, so that
// a lane's 8-byte reads of one row hit 8 distinct bank groups) through four
// buffers per warp -- two chunks ahead in flight, one being consumed, one
// receiving results (in place) before its TMA store.  Boxes beyond the system
// (or below row 0) read as zeros.  16-row boxes read 128 bytes of each system
// per DRAM burst instead of 64, with fewer warps per SM.
#pragma once
#include "jw_stream.cuh"

namespace pfb {

// Buffers per warp: four (two chunks ahead in flight); three for 16-row
// boxes above four steps (one chunk of 4 KB ahead), so that 14-15 warps fit
// beside the larger step tables instead of 9-10.
__host__ __device__ constexpr int seq_nbufs(int K, int CH) { return (CH == 16 && K > 4) ? 3 : 4; }
__host__ __device__ constexpr int seq_buf_bytes(int CH) { return CH * 32 * 8; }
// threads per CTA: 24 warps (85 registers a thread) for K <= 4 with 8-row
// boxes, else 16 warps (128 registers; 16-row boxes leave shared memory for
// about 12 warps anyway)
template <int K, int CH>
struct SeqThreads {
    static constexpr int v = (K > 4 || CH > 8) ? 512 : 768;
};

// Shared table: per step s and row i the pair {o, q} (matvec off-diagonal,
// solve band) at [s*Mtab + i], then the diagonal of the one step that applies
// it at [i] of a second plane.
__host__ __device__ constexpr size_t seq_table_bytes(int K, int64_t Mtab)
{
    return ((size_t)K * Mtab * 16 + (size_t)Mtab * 8 + 1023) / 1024 * 1024;
}
__host__ __device__ constexpr size_t seq_smem_bytes(int K, int64_t Mtab, int NW, int CH)
{
    return 1024 + seq_table_bytes(K, Mtab) + (size_t)NW * seq_nbufs(K, CH) * seq_buf_bytes(CH) +
           (size_t)NW * seq_nbufs(K, CH) * 8;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];\n" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, uint32_t src)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(map),
                 "r"(x), "r"(y), "r"(src)
                 : "memory");
}

// UB: 1 ascending sweep (upper matvec, lower solve), 0 descending.
// K: the number of steps (compiled per K, so the step loop unrolls exactly
// and the step that applies the matvec diagonal -- the first for UB 1, the
// last for UB 0 -- is known at compile time).  CH: rows per box (8 or 16).
template <int UB, bool MV, bool SV, int K, int CH>
__global__ void __launch_bounds__(SeqThreads<K, CH>::v) jw_steps_seq_kernel(const __grid_constant__ CUtensorMap tm_in,
                                                                      const __grid_constant__ CUtensorMap tm_out,
                                                                      const __grid_constant__ JwSteps S, const JwIO io)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int kSeqChunk = CH, kSeqBufBytes = seq_buf_bytes(CH), kSeqBufs = seq_nbufs(K, CH);
    constexpr int CM = CH - 1;                  // row within a chunk: & CM
    constexpr int CS = CH == 16 ? 4 : 3;        // chunk of a sweep position: >> CS
    constexpr int ROWB = CH * 8;                // bytes of a system's row in a box
    constexpr int KMAX = K;
    const int NW = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int M0 = (int)S.M_in, Mout = (int)S.M_out;
    const int Mtab = UB ? M0 : Mout;  // rows of the widest step

    unsigned char* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    double2* tabA = reinterpret_cast<double2*>(base);
    double* tabD = reinterpret_cast<double*>(base + (size_t)K * Mtab * 16);
    unsigned char* bufs = base + seq_table_bytes(K, Mtab) + (size_t)warp * kSeqBufs * kSeqBufBytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + seq_table_bytes(K, Mtab) + (size_t)NW * kSeqBufs * kSeqBufBytes) +
                     warp * kSeqBufs;

    // ---- coefficient table (rows at or beyond a step's M_s are never read)
    // the step that applies the matvec diagonal (JwStepDesc.diag)
    constexpr int dstep = MV ? (UB ? 0 : K - 1) : -1;
    for (int e = threadIdx.x; e < K * Mtab; e += blockDim.x) {
        const int s = e / Mtab, i = e - s * Mtab;
        const JwStepDesc& d = S.st[s];
        double o = 0.0, q = 0.0, dv = 1.0;
        if (i < d.M) {
            int pos = i;
            if (S.perm) {
                const int r = (int)d.perm_r, t = i / r, j = i - t * r, m = (int)d.perm_m;
                pos = t + ((j < m) ? j * (int)d.perm_ceil : m * (int)d.perm_ceil + (j - m) * (int)d.perm_floor);
            }
            if (MV) {
                if (d.diag) dv = __ldg(d.bands + d.off_md + pos);
                if (UB || i >= 1) o = __ldg(d.bands + d.off_mo + pos);
            }
            if (SV) {
                if (UB) q = (i >= 1) ? __ldg(d.bands + d.off_sl + pos) : 0.0;
                else q = __ldg(d.bands + d.off_su + pos);
            }
        }
        tabA[e] = make_double2(o, q);
        if (s == dstep) tabD[i] = dv;
    }
    if (lane < kSeqBufs) mbar_init(smem_u32(&bars[lane]), 1);
    mbar_init_fence();
    __syncthreads();

    // ---- sweep geometry (sweep position p <-> row): ascending p = row;
    // descending p = R0 - row with R0 the top row of the top chunk.  At sweep
    // time tau = p - 1 step s works at sweep position tau - s.
    const int R0 = UB ? 0 : ((Mout + kSeqChunk - 1) / kSeqChunk) * kSeqChunk - 1;
    const int pend = UB ? M0 : R0 + K;  // last input sweep position
    const int NK = pend / kSeqChunk + 1;
    const int cT = UB ? 0 : R0 / kSeqChunk;
    auto chunk_row0 = [&](int k) -> int { return UB ? k * kSeqChunk : (cT - k) * kSeqChunk; };
    const int lo = io.iz0 > 0 ? (int)io.iz0 : 0;          // rows read as data: [lo, hi)
    const int hi = io.iz1 < M0 ? (int)io.iz1 : M0;
    const int sw = CH == 16 ? (lane & 7) : ((lane >> 1) & 3);
    const double sC = S.scaleC;
    int Ms[KMAX];
#pragma unroll
    for (int s = 0; s < KMAX; ++s) Ms[s] = s < K ? (int)S.st[s].M : 0;
    const int64_t nblk = (io.nsys + 31) / 32;
    const uint32_t bufs_u = smem_u32(bufs);
    uint32_t seq = 0;  // chunk loads issued by this warp so far (buffer seq % kSeqBufs)
    bool ok = true;

    auto lds = [](uint32_t a) -> double {
        double v;
        asm volatile("ld.shared.f64 %0, [%1];\n" : "=d"(v) : "r"(a));
        return v;
    };
    auto lds2 = [](uint32_t a) -> double2 {
        double2 v;
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "r"(a));
        return v;
    };
    auto sts = [](uint32_t a, double v) { asm volatile("st.shared.f64 [%0], %1;\n" ::"r"(a), "d"(v) : "memory"); };
    // byte offset of box row rb (0 .. CH-1) of this lane's system in a buffer
    auto lane_off = [&](int rb) -> uint32_t {
        return (uint32_t)(lane * ROWB + ((((rb >> 1) ^ sw)) << 4) + ((rb & 1) << 3));
    };
    auto buf_of = [&](int k) -> uint32_t { return bufs_u + ((seq + (uint32_t)k) % kSeqBufs) * kSeqBufBytes; };
    auto issue = [&](int k, int sys0) {
        const uint32_t b = (seq + (uint32_t)k) % kSeqBufs;
        const uint32_t bar = smem_u32(&bars[b]);
        mbar_arrive_expect_tx(bar, kSeqBufBytes);
        tma_load_2d(bufs_u + b * kSeqBufBytes, &tm_in, chunk_row0(k), sys0, bar);
    };
    // A TMA store clips rows beyond M_out in 16-byte units: with M_out odd the
    // row after the last result would be written too.  The chunk holding an
    // odd last row is therefore written back with plain stores.
    auto store_chunk = [&](int k, int sys0) {
        const int r0 = chunk_row0(k);
        if ((Mout & 1) && r0 + kSeqChunk > Mout) {
            const int64_t y = (int64_t)sys0 + lane;
            if (y < io.nsys) {
                double* dst = io.out + io.out_off + y * io.out_stride;
                for (int rb = 0; rb < kSeqChunk && r0 + rb < Mout; ++rb) dst[r0 + rb] = lds(buf_of(k) + lane_off(rb));
            }
            return;
        }
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
            tma_store_2d(&tm_out, r0, sys0, buf_of(k));
            bulk_commit();
        }
    };
    const uint32_t tabA_u = smem_u32(tabA), tabD_u = smem_u32(tabD);

    for (int64_t blk = (int64_t)blockIdx.x * NW + warp; blk < nblk && ok; blk += (int64_t)gridDim.x * NW) {
        const int sys0 = (int)(blk * 32);
        if (lane == 0) {
            bulk_wait_read_all();  // the previous block's stores have read their buffers
            for (int k = 0; k < kSeqBufs - 1 && k < NK; ++k) issue(k, sys0);
        }
        __syncwarp();
        double xa[KMAX], zp[KMAX];
#pragma unroll
        for (int s = 0; s < KMAX; ++s) {
            xa[s] = 0.0;
            zp[s] = 0.0;
        }
        for (int k = 0; k < NK; ++k) {
            // chunk k: its load was issued kSeqBufs - 2 chunks ahead (or
            // before the sweep)
            if (lane == 0 && k >= 1) {
                // chunk k-2's store (issued during chunk k-1) has read the
                // buffer that chunk k + kSeqBufs - 2 takes
                bulk_wait_read_all();
                if (k + kSeqBufs - 2 < NK) issue(k + kSeqBufs - 2, sys0);
            }
            const uint32_t b = (seq + (uint32_t)k) % kSeqBufs;
            bool w = mbar_wait_bounded(smem_u32(&bars[b]), ((seq + (uint32_t)k) / kSeqBufs) & 1);
            w = __all_sync(FULL, w);
            if (!w) {
                if (lane == 0) atomicOr(&g_stream_status, kStatusWaitTimeout);
                ok = false;
                break;
            }
            const int rb = chunk_row0(k), p0 = k * kSeqChunk;
            const uint32_t cbuf = buf_of(k), pbuf = buf_of(k - 1);
            // steady chunk: every step active on rows 1 <= i < M_s, all input
            // rows inside the keep-window, every result row written
            const bool steady = UB ? (p0 >= K + 1 && p0 + CM < M0 && rb >= lo && rb + CH <= hi)
                                   : (p0 >= K + 1 && p0 + CM <= R0 && p0 >= R0 - M0 + 2 && p0 >= R0 - Mout + K + 1 &&
                                      rb >= lo && rb + CH <= hi);
            if (steady) {
                double vin[kSeqChunk];
#pragma unroll
                for (int u = 0; u < CH / 2; ++u) {
                    const double2 w2 = lds2(cbuf + lane * ROWB + ((u ^ sw) << 4));
                    if (UB) {
                        vin[2 * u] = w2.x;
                        vin[2 * u + 1] = w2.y;
                    } else {
                        vin[CM - 2 * u] = w2.x;
                        vin[CM - 1 - 2 * u] = w2.y;
                    }
                }
                // table row of step s at o = 0 (ascending: p0 - 1 - s;
                // descending: R0 - p0 + 1 + s); rows move by +-1 per o
                uint32_t ta[KMAX];
#pragma unroll
                for (int s = 0; s < KMAX; ++s)
                    ta[s] = tabA_u + (uint32_t)((s * Mtab + (UB ? p0 - 1 - s : R0 - p0 + 1 + s)) * 16);
                const uint32_t td = tabD_u + (uint32_t)((UB ? p0 - 1 - dstep : R0 - p0 + 1 + dstep) * 8);
#pragma unroll
                for (int o = 0; o < kSeqChunk; ++o) {
                    double v = vin[o];
#pragma unroll
                    for (int s = 0; s < KMAX; ++s) {
                        if (s < K) {
                            const double2 c = lds2(ta[s] + (UB ? 16 * o : -16 * o));
                            double y = xa[s];
                            if (MV && s == dstep) y *= lds(td + (UB ? 8 * o : -8 * o));
                            // z = (y - q z_prev) + o v: the part that does not
                            // depend on the step before is formed first, so
                            // the chain through the K steps is one FMA a step
                            if (SV) y = __fma_rn(-c.y, zp[s], y);
                            const double z = MV ? __fma_rn(c.x, v, y) : y;
                            zp[s] = z;
                            xa[s] = v;
                            v = z;
                        }
                    }
                    const int oo = o - K;  // result position relative to this chunk
                    const int qo = oo & CM;
                    sts((oo >= 0 ? cbuf : pbuf) + lane_off(UB ? qo : CM - qo), v);
                    if (o == K - 1) store_chunk(k - 1, sys0);
                }
                continue;
            }
#pragma unroll
            for (int o = 0; o < kSeqChunk; ++o) {
                const int p = p0 + o;  // input sweep position
                if (p > pend) break;
                const int rbx = UB ? o : kSeqChunk - 1 - o;
                const int row = rb + rbx;
                double v = 0.0;
                if (row >= lo && row < hi) v = lds(cbuf + lane_off(rbx));
                if (p == 0) {
                    xa[0] = v;
                    continue;
                }
                bool out = true;
#pragma unroll
                for (int s = 0; s < KMAX; ++s) {
                    if (s >= K) break;
                    const int ps = p - 1 - s;
                    if (ps < 0) {
                        if (ps == -1) xa[s] = v;
                        out = false;
                        break;
                    }
                    const int i = UB ? ps : R0 - ps;
                    double z;
                    if (i < 0) {
                        z = 0.0;
                    } else if (i < Ms[s]) {
                        const double2 c = lds2(tabA_u + (uint32_t)((s * Mtab + i) * 16));
                        double y = xa[s];
                        if (MV && s == dstep) y *= lds(tabD_u + (uint32_t)(i * 8));
                        if (SV) y = __fma_rn(-c.y, zp[s], y);
                        z = MV ? __fma_rn(c.x, v, y) : y;
                    } else {
                        z = xa[s];
                    }
                    zp[s] = z;
                    xa[s] = v;
                    v = (SV && i == 0) ? sC * z : z;
                }
                if (!out) continue;
                // v: result of the last step at sweep position q = p - K
                const int q = p - K;
                const int qk = q >> CS, qo = q & CM;
                const int qrb = UB ? qo : kSeqChunk - 1 - qo;
                const int orow = chunk_row0(qk) + qrb;
                if (orow >= 0 && orow < Mout) sts(buf_of(qk) + lane_off(qrb), v);
                if (qo == kSeqChunk - 1 || (UB && orow == Mout - 1)) store_chunk(qk, sys0);
            }
        }
        seq += (uint32_t)NK;
    }
    if (lane == 0) bulk_wait_all();
}

}  // namespace pfb
