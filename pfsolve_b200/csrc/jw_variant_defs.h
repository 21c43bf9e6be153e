// jw_variant_defs.h -- helpers and macros that instantiate JW-step kernel
// variants into the per-file variant tables.
#pragma once
#include "dd_kernel.cuh"
#include "jw_kernel.cuh"
#include "jw_variants.h"

namespace pfb {

template <class C>
inline size_t smem_fn(int W, int G)
{
    return jw_smem_bytes<C>(W, G);
}

template <class C>
inline void launch_fn(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const JwOperator& op, const JwIO& io, int W)
{
    jw_step_kernel<C><<<grid, block, smem, st>>>(op, io, W);
}

#define PFB_VT(R, KL, KU, SV, LIN, LOUT, SC, P, T)                                                     \
    JwVariant{R, KL, KU, SV, LIN, LOUT, SC, P, T, JwCfg<R, KL, KU, SV, LIN, LOUT, SC, P, T>::kMaxThreads,  \
              (const void*)&jw_step_kernel<JwCfg<R, KL, KU, SV, LIN, LOUT, SC, P, T>>,                    \
              &smem_fn<JwCfg<R, KL, KU, SV, LIN, LOUT, SC, P, T>>, &launch_fn<JwCfg<R, KL, KU, SV, LIN, LOUT, SC, P, T>>}
#define PFB_VP(R, KL, KU, SV, LIN, LOUT, SC, P) PFB_VT(R, KL, KU, SV, LIN, LOUT, SC, P, false)
#define PFB_V(R, KL, KU, SV, LIN, LOUT, SC) PFB_VP(R, KL, KU, SV, LIN, LOUT, SC, PREC_F64)
// coefficient-table variants (FP64), rows per thread 4 and 8
#define PFB_T2(KL, KU, SV, LIN, LOUT, SC) \
    PFB_VT(4, KL, KU, SV, LIN, LOUT, SC, PREC_F64, true), PFB_VT(8, KL, KU, SV, LIN, LOUT, SC, PREC_F64, true)

// double-double variants: PREC 2 = dd storage, PREC 3 = dd arithmetic on FP64 storage
template <class C>
inline size_t dd_smem_fn(int W, int G)
{
    return dd_smem_bytes<C>(W, G);
}
template <class C>
inline void dd_launch_fn(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const JwOperator& op, const JwIO& io,
                         int W)
{
    jw_dd_kernel<C><<<grid, block, smem, st>>>(op, io, W);
}
#define PFB_DDV(R, KL, KU, SV, MEM)                                                                     \
    JwVariant{R, KL, KU, SV, LAY_REAL, LAY_REAL, 0, (MEM) ? 2 : 3, 0, 256,                              \
              (const void*)&jw_dd_kernel<DdCfg<R, KL, KU, SV, MEM>>, &dd_smem_fn<DdCfg<R, KL, KU, SV, MEM>>, \
              &dd_launch_fn<DdCfg<R, KL, KU, SV, MEM>>}
template <class C>
inline void dd_tbl_launch_fn(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const JwOperator& op,
                             const JwIO& io, int W)
{
    jw_dd_tbl_kernel<C><<<grid, block, smem, st>>>(op, io, W);
}
// table form (TBL = 1): coefficients, chunk products and scan multipliers in
// shared memory
#define PFB_DDT(R, KL, KU, SV, MEM)                                                                               \
    JwVariant{R, KL, KU, SV, LAY_REAL, LAY_REAL, 0, (MEM) ? 2 : 3, 1, 256,                                        \
              (const void*)&jw_dd_tbl_kernel<DdCfg<R, KL, KU, SV, MEM, true>>,                                      \
              &dd_smem_fn<DdCfg<R, KL, KU, SV, MEM, true>>, &dd_tbl_launch_fn<DdCfg<R, KL, KU, SV, MEM, true>>}
#define PFB_DD(KL, KU, SV)                                                                                 \
    PFB_DDV(4, KL, KU, SV, true), PFB_DDV(8, KL, KU, SV, true), PFB_DDV(4, KL, KU, SV, false),               \
        PFB_DDV(8, KL, KU, SV, false), PFB_DDT(8, KL, KU, SV, true), PFB_DDT(16, KL, KU, SV, true),          \
        PFB_DDT(8, KL, KU, SV, false), PFB_DDT(16, KL, KU, SV, false)

// Rows-per-thread choices for the single-application (drop-in) variants.
#define PFB_R4(KL, KU, SV, LIN, LOUT, SC) \
    PFB_V(2, KL, KU, SV, LIN, LOUT, SC), PFB_V(4, KL, KU, SV, LIN, LOUT, SC), PFB_V(8, KL, KU, SV, LIN, LOUT, SC), \
        PFB_V(16, KL, KU, SV, LIN, LOUT, SC)
#define PFB_R2(KL, KU, SV, LIN, LOUT, SC) PFB_V(4, KL, KU, SV, LIN, LOUT, SC), PFB_V(8, KL, KU, SV, LIN, LOUT, SC)
#define PFB_M2(KL, KU, SV, LIN, LOUT, SC) \
    PFB_VP(4, KL, KU, SV, LIN, LOUT, SC, PREC_MIXED), PFB_VP(8, KL, KU, SV, LIN, LOUT, SC, PREC_MIXED)
// the same rows-per-thread choices in a given precision (the FP32-storage ones)
#define PFB_R4P(KL, KU, SV, LIN, LOUT, SC, P)                                                                \
    PFB_VP(2, KL, KU, SV, LIN, LOUT, SC, P), PFB_VP(4, KL, KU, SV, LIN, LOUT, SC, P),                          \
        PFB_VP(8, KL, KU, SV, LIN, LOUT, SC, P), PFB_VP(16, KL, KU, SV, LIN, LOUT, SC, P)
#define PFB_R2P(KL, KU, SV, LIN, LOUT, SC, P) PFB_VP(4, KL, KU, SV, LIN, LOUT, SC, P), PFB_VP(8, KL, KU, SV, LIN, LOUT, SC, P)
// every application kind of the FP32-storage precisions: the JW application
// on real systems, the dgbmv application with KL, KU <= 2, and the fused
// chains the FP64 tables hold
#define PFB_F32_KINDS(P)                                                                                      \
    PFB_R4P(0, 0, SV_TRI, LAY_REAL, LAY_REAL, false, P), PFB_R4P(0, 1, SV_LOWER, LAY_REAL, LAY_REAL, false, P), \
        PFB_R4P(0, 1, SV_NONE, LAY_REAL, LAY_REAL, false, P), PFB_R4P(0, 0, SV_LOWER, LAY_REAL, LAY_REAL, false, P), \
        PFB_R4P(1, 0, SV_UPPER, LAY_REAL, LAY_REAL, false, P), PFB_R4P(1, 0, SV_NONE, LAY_REAL, LAY_REAL, false, P), \
        PFB_R4P(0, 0, SV_UPPER, LAY_REAL, LAY_REAL, false, P), PFB_R2P(1, 1, SV_NONE, LAY_REAL, LAY_REAL, false, P), \
        PFB_R2P(2, 2, SV_NONE, LAY_REAL, LAY_REAL, false, P), PFB_R2P(0, 2, SV_NONE, LAY_REAL, LAY_REAL, false, P), \
        PFB_R2P(2, 0, SV_NONE, LAY_REAL, LAY_REAL, false, P), PFB_R2P(1, 2, SV_NONE, LAY_REAL, LAY_REAL, false, P), \
        PFB_R2P(2, 1, SV_NONE, LAY_REAL, LAY_REAL, false, P), PFB_R2P(0, 0, SV_NONE, LAY_REAL, LAY_REAL, false, P), \
        PFB_R2P(1, 1, SV_UPPER, LAY_REAL, LAY_REAL, false, P), PFB_R2P(1, 1, SV_LOWER, LAY_REAL, LAY_REAL, false, P), \
        PFB_R2P(1, 1, SV_TRI, LAY_REAL, LAY_REAL, false, P), PFB_R2P(2, 2, SV_TRI, LAY_REAL, LAY_REAL, false, P),   \
        PFB_R2P(0, 0, SV_TRI, LAY_REAL, LAY_REAL, true, P), PFB_R2P(1, 1, SV_UPPER, LAY_REAL, LAY_REAL, true, P),   \
        PFB_R2P(2, 2, SV_TRI, LAY_XXII, LAY_PACKED, false, P), PFB_R2P(2, 2, SV_TRI, LAY_XXII, LAY_PACKED, true, P), \
        PFB_R2P(0, 0, SV_TRI, LAY_XXII, LAY_PACKED, false, P), PFB_R2P(1, 1, SV_UPPER, LAY_XXII, LAY_PACKED, true, P), \
        PFB_R2P(1, 1, SV_UPPER, LAY_XXII, LAY_PACKED, false, P), PFB_R2P(0, 0, SV_UPPER, LAY_XXII, LAY_PACKED, true, P)


}  // namespace pfb
