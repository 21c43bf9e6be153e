// steps_variants.cu -- instantiations of the K-step JW kernel (jw_steps.cuh):
// the six defined operator kinds of upperBanded 0/1 (jw_type 10, 11, 12) and
// the tridiagonal kind of upperBanded 2 (jw_type 13), at 4, 8 and 16 rows per
// thread.
#include "jw_steps.cuh"
#include "jw_variants.h"

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

}  // namespace pfb
