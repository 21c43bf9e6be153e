// jw_variants.h -- host-side table of precompiled JW-step kernel variants.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "jw_types.h"

namespace pfb {

using JwKernelFn = void (*)(JwOperator, JwIO, int);

struct JwVariant {
    int R, KL, KU, SV, LIN, LOUT, SCALE, PREC, TBL;
    int max_threads;                   // launch bound of the entry
    const void* func;                  // __global__ entry (for attributes / occupancy)
    size_t (*smem_bytes)(int W, int G);
    void (*launch)(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const JwOperator& op, const JwIO& io, int W);
};

// Find a variant; nullptr when that combination was not compiled.
const JwVariant* find_jw_variant(int R, int KL, int KU, int SV, int LIN, int LOUT, int SCALE, int PREC = 0,
                                int TBL = 0);

// Persistent uneven-batch kernels (one per operator shape).
struct BatchVariant {
    int R, KL, KU, SV, LIN, LOUT, SCALE, PREC;
    const void* func;
    size_t (*smem_bytes)(int W, int G);
    void (*launch)(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const BatchEntryDev* entries,
                   const WorkItem* items, int nitems, unsigned int* counter, int W);
};
const BatchVariant* find_batch_variant(int R, int KL, int KU, int SV, int LIN, int LOUT, int SCALE, int PREC);

// Uneven batches of bidiagonal steps (V*A within rows i-1..i+1, XXII in,
// packed complex out, FP64): one complex system per lane, each system's rows
// in one sweep, items of up to 32 systems per warp, NBUF chunks of 8 rows
// staged per warp, NW warps per CTA.  `coefs` launches the pre-pass that
// writes every entry's coefficient rows (48 bytes each, batch_seq_rows(M) per
// entry from row coef_off) before the sweep.
struct alignas(64) BatchSeqEntry {
    CUtensorMap in[2];  // {2 in_stride, nsys} doubles, boxes 8 x 32 (64-byte swizzle) and 16 x 32 (128-byte)
    CUtensorMap out;    // {2 M, nsys} doubles at row pitch 16 out_stride bytes, box 16 x 32, 128-byte swizzle
    int64_t coef_off;   // first coefficient row of the entry
    int tma_in;         // input 16-byte aligned with in_stride >= M: TMA boxes (else 8-byte cp.async)
    int pad[13];
};
// CH rows per chunk (8 or 16).
struct BatchSeqVariant {
    int SV, CH, NBUF, NW;
    const void* func;
    void (*launch)(dim3 grid, size_t smem, cudaStream_t st, const BatchEntryDev* entries, const BatchSeqEntry* seq,
                   const double* coefs, const WorkItem* items, int nitems, unsigned int* counter);
    void (*coefs)(int nentries, cudaStream_t st, const BatchEntryDev* entries, const BatchSeqEntry* seq,
                  double* coefs);
};
const BatchSeqVariant* find_batch_seq_variant(int SV, int shape);  // shape: index into the compiled shapes
constexpr int kBatchSeqShapes = 3;
int64_t batch_seq_rows(int64_t M);  // coefficient rows of an entry of M rows
// Tensor maps of one entry; false when its output cannot take TMA stores.
bool encode_batch_seq_maps(const JwIO& io, BatchSeqEntry* e);
unsigned batch_status_fetch_clear();  // the sweep batch kernel's waits
size_t batch_seq_smem(const BatchSeqVariant* v);  // dynamic shared memory of a launch

// Streaming variants (TMA-staged systems, R rows per thread, W warps per
// system).  IB / IBO: 16-byte units per swizzle row of the input / output
// layout (the TMA box's inner extent).
struct StreamVariant {
    int R, W, KL, KU, SV, LIN, LOUT, SCALE, PREC;
    int max_threads;
    const void* func;
    size_t (*smem_bytes)(int G, int NB);  // G groups of NB staging buffers
    int IB, IBO;
    void (*launch)(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const CUtensorMap* in, const CUtensorMap* out,
                   const JwOperator& op, const JwIO& io);
    int ALT = 0;  // ALT stride-2 mode: one staged row set holds two systems (its even and odd rows)
};
const StreamVariant* find_stream_variant(int R, int W, int KL, int KU, int SV, int LIN, int LOUT, int SCALE,
                                        int PREC, int ALT = 0);
// Tensor maps of a launch's input and output rows; false when the buffers'
// alignment, strides or M do not allow the streaming layout.
bool encode_stream_maps(const StreamVariant* v, const JwIO& io, CUtensorMap* in, CUtensorMap* out);
// es: bytes per stored value (8: FP64, 4: FP32).
bool encode_row_maps(int R, int LIN, int LOUT, int IB, int IBO, const JwIO& io, CUtensorMap* in, CUtensorMap* out,
                     int es = 8);

// Long-system variants: one cluster of C CTAs per system, each CTA a slice of
// 32*W*R rows (real systems, FP64).
struct ClusterVariant {
    int R, W, C, KL, KU, SV;
    const void* func;
    size_t smem_bytes;
    int IB, IBO;
    // grid: clusters * C CTAs; returns the launch error
    cudaError_t (*launch)(int clusters, size_t smem, cudaStream_t st, const CUtensorMap* in, const CUtensorMap* out,
                          const JwOperator& op, const JwIO& io);
    int (*max_clusters)(size_t smem);  // clusters that fit the device at once (0: none)
};
const ClusterVariant* find_cluster_variant(int C, int KL, int KU, int SV);

// Long systems over slices of S = 32 W R rows, G systems in flight per CTA;
// launch = the table passes (two for a tridiagonal solve), then the single
// pass (`single`: one cooperative launch whose CTAs wait for the other slices
// of each system, up to kLgMaxSlices slices) or pass 1, the carry kernel
// (solves only) and pass 2 on the stream.  red: nsys * NS records of 8
// doubles, cst: NS records of 8 doubles, tab: NS slice tables of tbl_bytes,
// flags: nsys * NS words (single pass; zero before the first launch),
// epoch: the launch's flag value (never 0, never repeated while flags live).
struct LongVariant {
    int R, W, G, KL, KU, SV, S;
    int IB, IBO;
    size_t tbl_bytes;
    cudaError_t (*launch)(int grid, cudaStream_t st, const CUtensorMap* in, const CUtensorMap* out,
                          const JwOperator& op, const JwIO& io, double* red, double* cst, double* tab, int NS,
                          unsigned* flags, unsigned epoch, bool single);
    int (*blocks_per_sm)(bool single);  // resident CTAs per SM of the single pass or the two (0: does not fit)
};
constexpr int kLongMaxSlices = 64;  // slices per system of the single pass
constexpr int kLongShapes = 4;  // compiled shapes per operator kind, in order of preference
const LongVariant* find_long_variant(int shape, int KL, int KU, int SV);

// The DCT step (dct.cu): type 2 or 3 of rows of 2^logn points (3 <= logn <=
// 12), with the plan's tables from dct_tables (twiddles, then the pre/post
// factors; 2N values of 16 bytes, one cudaMalloc).
cudaError_t dct_launch(int logn, int type, const DctIO& io, const double2* tw, const double2* pt, int num_sms,
                       cudaStream_t st);
cudaError_t dct_tables(int64_t N, double2** tables);
unsigned long_status_fetch_clear();
unsigned cluster_status_fetch_clear();
// Status word of the streaming kernels' bounded waits since the last call
// (0: none timed out); reading it synchronises with the device.
unsigned stream_status_fetch_clear();
unsigned steps_status_fetch_clear();  // the K-step sweep kernel's waits

// K consecutive JW steps in one kernel (real FP64 systems; R rows per thread,
// W warps per system given at launch).  MV: the steps have a matvec.
struct StepsVariant {
    int R, KL, KU, SV, MV;
    const void* func;
    size_t (*smem_bytes)(int K, int W, int G);
    void (*launch)(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const JwSteps& S, const JwIO& io, int W);
};
const StepsVariant* find_steps_variant(int R, int KL, int KU, int SV, int MV);

// K bidiagonal steps, one system per lane, all steps in one sweep (UB 1:
// ascending rows, 0: descending), compiled for K = KMAX steps; systems staged by TMA boxes of
// 8 rows x 32 systems.
struct SeqStepsVariant {
    int UB, MV, SV, KMAX, CH;  // CH: rows per TMA box (8 or 16)
    int max_threads;
    const void* func;
    void (*launch)(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const CUtensorMap* in, const CUtensorMap* out,
                   const JwSteps& S, const JwIO& io);
};
const SeqStepsVariant* find_seq_steps_variant(int UB, int MV, int SV, int K, int CH);
size_t seq_steps_smem_bytes(int K, int64_t Mtab, int NW, int CH);
// 2-D tensor maps {rows, systems} of a K-step launch's right-hand sides: M_in
// rows read, M_out rows written, boxes of CH (8 or 16) rows x 32 systems;
// false when the buffers' alignment or stride does not allow them.
bool encode_seq_maps(const JwIO& io, int64_t M_in, int64_t M_out, int CH, CUtensorMap* in, CUtensorMap* out);

// Standalone kernels of the block and generic-bandwidth dgbmv applications.
struct BlockArgs {
    const double* in;
    double* out;
    int64_t size0, size1;
    int64_t in_off, in_stride, out_off, out_stride;
    int64_t iz0, iz1, oz0, oz1;
    int layout;  // block % 10
    int accumulate;
    int scale_kind, lshift;
    double s;
    int skip_read;
    int f32;  // FP32 storage (in and out hold FP32 values)
};
void launch_block(const BlockArgs& a, cudaStream_t st, int num_sms);

struct DgbmvArgs {
    const double* A;
    double* x;
    int64_t M, nsys, off_A, off_x, stride;
    int lda, ku;
    int64_t iz0, iz1, oz0, oz1;
    uint64_t skip;  // ALT_dgbmv: bit j set drops band j
    int f32;        // FP32 storage (A and x hold FP32 values)
};
void launch_dgbmv_generic(const DgbmvArgs& a, cudaStream_t st, int num_sms);

}  // namespace pfb
