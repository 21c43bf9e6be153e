// stream_variant_defs.h -- helpers and macros that instantiate streaming
// JW-step kernel variants into the per-file variant tables.  Every file that
// includes it gets its own copy of the device status word (g_stream_status)
// and defines an accessor for it.
#pragma once
#include <cuda.h>

#include "jw_stream.cuh"
#include "jw_variants.h"

namespace pfb {

template <class C>
inline size_t st_smem_fn(int G, int NB)
{
    return st_smem_bytes<C>(G, NB);
}

template <class C>
inline void st_launch_fn(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const CUtensorMap* in,
                         const CUtensorMap* out, const JwOperator& op, const JwIO& io)
{
    jw_stream_kernel<C><<<grid, block, smem, st>>>(*in, *out, op, io);
}

#define PFB_SVP(R, W, KL, KU, SV, LIN, LOUT, SC, P)                                                     \
    StreamVariant{R, W, KL, KU, SV, LIN, LOUT, SC, P, StCfg<R, W, KL, KU, SV, LIN, LOUT, SC, P>::kMaxThreads, \
                  (const void*)&jw_stream_kernel<StCfg<R, W, KL, KU, SV, LIN, LOUT, SC, P>>,                 \
                  &st_smem_fn<StCfg<R, W, KL, KU, SV, LIN, LOUT, SC, P>>,                                    \
                  StCfg<R, W, KL, KU, SV, LIN, LOUT, SC, P>::IB, StCfg<R, W, KL, KU, SV, LIN, LOUT, SC, P>::IBO, \
                  &st_launch_fn<StCfg<R, W, KL, KU, SV, LIN, LOUT, SC, P>>}
#define PFB_SV(R, W, KL, KU, SV, LIN, LOUT, SC) PFB_SVP(R, W, KL, KU, SV, LIN, LOUT, SC, PREC_F64)
// ALT stride-2 mode: real FP64 row sets, each holding two systems
#define PFB_SVA(R, W, KL, KU, SV)                                                                              \
    StreamVariant{R, W, KL, KU, SV, LAY_REAL, LAY_REAL, false, PREC_F64,                                      \
                  StCfg<R, W, KL, KU, SV, LAY_REAL, LAY_REAL, false, PREC_F64, 1>::kMaxThreads,                \
                  (const void*)&jw_stream_kernel<StCfg<R, W, KL, KU, SV, LAY_REAL, LAY_REAL, false, PREC_F64, 1>>, \
                  &st_smem_fn<StCfg<R, W, KL, KU, SV, LAY_REAL, LAY_REAL, false, PREC_F64, 1>>,                 \
                  StCfg<R, W, KL, KU, SV, LAY_REAL, LAY_REAL, false, PREC_F64, 1>::IB,                          \
                  StCfg<R, W, KL, KU, SV, LAY_REAL, LAY_REAL, false, PREC_F64, 1>::IBO,                         \
                  &st_launch_fn<StCfg<R, W, KL, KU, SV, LAY_REAL, LAY_REAL, false, PREC_F64, 1>>, 1}
// 8, 16 and 32 rows per thread, 1, 2 and 4 warps per row set (M <= 4096)
#define PFB_SALT(KL, KU, SV)                                                                                  \
    PFB_SVA(8, 1, KL, KU, SV), PFB_SVA(8, 2, KL, KU, SV), PFB_SVA(8, 4, KL, KU, SV), PFB_SVA(16, 1, KL, KU, SV), \
        PFB_SVA(16, 2, KL, KU, SV), PFB_SVA(16, 4, KL, KU, SV), PFB_SVA(32, 1, KL, KU, SV),                    \
        PFB_SVA(32, 2, KL, KU, SV), PFB_SVA(32, 4, KL, KU, SV)
// real systems: 8 rows per thread (M <= 256, 512, 1024), 16 (M <= 512, 1024,
// 2048) and 32 (M <= 1024, 2048, 4096)
#define PFB_SREALP(KL, KU, SV, P)                                                                        \
    PFB_SVP(8, 1, KL, KU, SV, LAY_REAL, LAY_REAL, false, P), PFB_SVP(8, 2, KL, KU, SV, LAY_REAL, LAY_REAL, false, P),   \
        PFB_SVP(8, 4, KL, KU, SV, LAY_REAL, LAY_REAL, false, P), PFB_SVP(16, 1, KL, KU, SV, LAY_REAL, LAY_REAL, false, P), \
        PFB_SVP(16, 2, KL, KU, SV, LAY_REAL, LAY_REAL, false, P), PFB_SVP(16, 4, KL, KU, SV, LAY_REAL, LAY_REAL, false, P), \
        PFB_SVP(32, 1, KL, KU, SV, LAY_REAL, LAY_REAL, false, P), PFB_SVP(32, 2, KL, KU, SV, LAY_REAL, LAY_REAL, false, P), \
        PFB_SVP(32, 4, KL, KU, SV, LAY_REAL, LAY_REAL, false, P)
#define PFB_SREAL(KL, KU, SV) PFB_SREALP(KL, KU, SV, PREC_F64)
// complex XXII right-hand sides written packed
#define PFB_SCPLXP(KL, KU, SV, SC, P)                                                                             \
    PFB_SVP(16, 1, KL, KU, SV, LAY_XXII, LAY_PACKED, SC, P), PFB_SVP(16, 2, KL, KU, SV, LAY_XXII, LAY_PACKED, SC, P), \
        PFB_SVP(32, 1, KL, KU, SV, LAY_XXII, LAY_PACKED, SC, P), PFB_SVP(32, 2, KL, KU, SV, LAY_XXII, LAY_PACKED, SC, P)
#define PFB_SCPLX(KL, KU, SV, SC) PFB_SCPLXP(KL, KU, SV, SC, PREC_F64)


// Status word of this translation unit's kernels: read and clear.
#define PFB_STREAM_STATUS_ACCESSOR(name)                                          \
    unsigned name()                                                               \
    {                                                                             \
        unsigned v = 0, zero = 0;                                                 \
        if (cudaMemcpyFromSymbol(&v, g_stream_status, sizeof(v)) != cudaSuccess) \
            return ~0u;                                                           \
        if (v) cudaMemcpyToSymbol(g_stream_status, &zero, sizeof(zero));          \
        return v;                                                                 \
    }

}  // namespace pfb
