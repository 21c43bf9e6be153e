// steps_variants.cu -- instantiations of the K-step JW kernels: the partition
// kernel (jw_steps.cuh) for the six defined operator kinds of upperBanded 0/1
// (jw_type 10, 11, 12) and the tridiagonal kind of upperBanded 2 (jw_type 13)
// at 4, 8 and 16 rows per thread; the one-system-per-lane sweep kernel
// (jw_steps_seq.cuh) for the six bidiagonal kinds with K up to 2, 4 or 8.
#include "jw_steps.cuh"
#include "jw_steps_seq.cuh"
#include "jw_variants.h"
#include "stream_variant_defs.h"

namespace pfb {

template <class C>
static size_t steps_smem_fn(int K, int W, int G)
{
    return ks_smem_bytes<C>(K, W, G);
}

template <class C>
static void steps_launch_fn(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const JwSteps& S, const JwIO& io,
                            int W)
{
    jw_steps_kernel<C><<<grid, block, smem, st>>>(S, io, W);
}

#define PFB_KS(R, KL, KU, SV, MV)                                                                        \
    StepsVariant{R, KL, KU, SV, MV, (const void*)&jw_steps_kernel<KsCfg<R, KL, KU, SV, MV>>,            \
                 &steps_smem_fn<KsCfg<R, KL, KU, SV, MV>>, &steps_launch_fn<KsCfg<R, KL, KU, SV, MV>>}
#define PFB_KS3(KL, KU, SV, MV) PFB_KS(4, KL, KU, SV, MV), PFB_KS(8, KL, KU, SV, MV), PFB_KS(16, KL, KU, SV, MV)

static const StepsVariant kStepsVariants[] = {
    PFB_KS3(0, 1, SV_LOWER, true),   // upperBanded 1, jw_type 10
    PFB_KS3(0, 1, SV_NONE, true),    // upperBanded 1, jw_type 11
    PFB_KS3(0, 0, SV_LOWER, false),  // upperBanded 1, jw_type 12
    PFB_KS3(1, 0, SV_UPPER, true),   // upperBanded 0, jw_type 10
    PFB_KS3(1, 0, SV_NONE, true),    // upperBanded 0, jw_type 11
    PFB_KS3(0, 0, SV_UPPER, false),  // upperBanded 0, jw_type 12
    PFB_KS3(0, 0, SV_TRI, true),     // upperBanded 2, jw_type 13
};

const StepsVariant* find_steps_variant(int R, int KL, int KU, int SV, int MV)
{
    for (const StepsVariant& v : kStepsVariants)
        if (v.R == R && v.KL == KL && v.KU == KU && v.SV == SV && v.MV == (MV ? 1 : 0)) return &v;
    return nullptr;
}

template <int UB, bool MV, bool SV, int K, int CH>
static void seq_launch_fn(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const CUtensorMap* in,
                          const CUtensorMap* out, const JwSteps& S, const JwIO& io)
{
    jw_steps_seq_kernel<UB, MV, SV, K, CH><<<grid, block, smem, st>>>(*in, *out, S, io);
}

#define PFB_SQC(UB, MV, SV, K, CH)                                                                            \
    SeqStepsVariant{UB, MV, SV, K, CH, SeqThreads<K, CH>::v, (const void*)&jw_steps_seq_kernel<UB, MV, SV, K, CH>, \
                    &seq_launch_fn<UB, MV, SV, K, CH>}
#define PFB_SQ(UB, MV, SV, K) PFB_SQC(UB, MV, SV, K, 8), PFB_SQC(UB, MV, SV, K, 16)
// one instance per step count, 2..8: 16-row boxes up to 6 steps (the default
// there), 8-row boxes at every count
#define PFB_SQ3(UB, MV, SV)                                                                               \
    PFB_SQ(UB, MV, SV, 2), PFB_SQ(UB, MV, SV, 3), PFB_SQ(UB, MV, SV, 4), PFB_SQ(UB, MV, SV, 5),            \
        PFB_SQ(UB, MV, SV, 6), PFB_SQC(UB, MV, SV, 7, 8), PFB_SQC(UB, MV, SV, 8, 8)

static const SeqStepsVariant kSeqVariants[] = {
    PFB_SQ3(1, true, true), PFB_SQ3(1, true, false), PFB_SQ3(1, false, true),
    PFB_SQ3(0, true, true), PFB_SQ3(0, true, false), PFB_SQ3(0, false, true),
};

const SeqStepsVariant* find_seq_steps_variant(int UB, int MV, int SV, int K, int CH)
{
    for (const SeqStepsVariant& v : kSeqVariants)
        if (v.UB == UB && v.MV == (MV ? 1 : 0) && v.SV == (SV ? 1 : 0) && K == v.KMAX && CH == v.CH) return &v;
    return nullptr;
}

size_t seq_steps_smem_bytes(int K, int64_t Mtab, int NW, int CH) { return seq_smem_bytes(K, Mtab, NW, CH); }

// status of the sweep kernel's bounded waits
PFB_STREAM_STATUS_ACCESSOR(steps_status_fetch_clear)

}  // namespace pfb
