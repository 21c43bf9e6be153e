// long_variants.cu -- instantiations of the two-pass long-system JW-step
// kernel (jw_long.cuh), their launch, and the status word of their waits.
#include <cuda.h>

#include "jw_long.cuh"
#include "jw_variants.h"
#include "plan.h"
#include "stream_variant_defs.h"

namespace pfb {

// The table passes, then either the single pass (a cooperative launch: every
// CTA resident, as its cross-CTA waits need) or pass 1, the carry kernel and
// pass 2.
template <class C>
static cudaError_t lg_launch_fn(int grid, cudaStream_t st, const CUtensorMap* in, const CUtensorMap* out,
                                const JwOperator& op, const JwIO& io, double* red, double* cst, double* tab, int NS,
                                unsigned* flags, unsigned epoch, bool single)
{
    const size_t smem = lg_smem_bytes<C>();
    if (C::SV == SV_TRI)
        jw_long_kernel<C, 3><<<NS, C::NT, smem, st>>>(*in, *out, op, io, red, cst, tab, NS, flags, epoch);
    jw_long_kernel<C, 0><<<NS, C::NT, smem, st>>>(*in, *out, op, io, red, cst, tab, NS, flags, epoch);
    if (single) {
        if (NS > kLgMaxSlices) return cudaErrorInvalidValue;
        CUtensorMap tin = *in, tout = *out;
        JwOperator o = op;
        JwIO i = io;
        int ns = NS;
        unsigned ep = epoch;
        void* args[] = {&tin, &tout, &o, &i, &red, &cst, &tab, &ns, &flags, &ep};
        const cudaError_t e = cudaLaunchCooperativeKernel((const void*)&jw_long_kernel<C, 4>, dim3((unsigned)grid),
                                                          dim3(C::NT), args, lg_smem_bytes<C, 3>(), st);
        if (e != cudaSuccess) return e;
        return cudaPeekAtLastError();
    }
    jw_long_kernel<C, 1><<<grid, C::NT, smem, st>>>(*in, *out, op, io, red, cst, tab, NS, flags, epoch);
    if (C::B::FWD || C::B::BWD)
        jw_long_carry_kernel<C::B::FWD, C::B::BWD>
            <<<(unsigned)((io.nsys + 127) / 128), 128, 0, st>>>(red, cst, NS, io.nsys);
    jw_long_kernel<C, 2><<<grid, C::NT, smem, st>>>(*in, *out, op, io, red, cst, tab, NS, flags, epoch);
    return cudaPeekAtLastError();
}

// resident CTAs per SM of the single pass (single) or of the two passes
// (0: does not fit)
template <class C>
static int lg_blocks_per_sm(bool single)
{
    const void* f3 = (const void*)&jw_long_kernel<C, 3>;
    const void* f0 = (const void*)&jw_long_kernel<C, 0>;
    if (!allow_max_smem(f3) || !allow_max_smem(f0)) return 0;
    int b1 = 0, b2 = 0;
    if (single) {
        const void* f4 = (const void*)&jw_long_kernel<C, 4>;
        int maxopt = 0, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (lg_smem_bytes<C, 3>() > (size_t)maxopt || !allow_max_smem(f4)) return 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, f4, C::NT, lg_smem_bytes<C, 3>()) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        return b1;
    }
    const size_t smem = lg_smem_bytes<C>();
    const void* f1 = (const void*)&jw_long_kernel<C, 1>;
    const void* f2 = (const void*)&jw_long_kernel<C, 2>;
    if (!allow_max_smem(f1) || !allow_max_smem(f2)) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, f1, C::NT, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, f2, C::NT, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return b1 < b2 ? b1 : b2;
}

#define PFB_LG(R, W, G, KL, KU, SV)                                                                    \
    LongVariant{R, W, G, KL, KU, SV, LgCfg<R, W, G, KL, KU, SV>::S, LgCfg<R, W, G, KL, KU, SV>::B::IB,     \
                LgCfg<R, W, G, KL, KU, SV>::B::IBO, LgCfg<R, W, G, KL, KU, SV>::B::TBL,                    \
                &lg_launch_fn<LgCfg<R, W, G, KL, KU, SV>>, &lg_blocks_per_sm<LgCfg<R, W, G, KL, KU, SV>>}
// (rows per thread, warps per slice, systems in flight per CTA): slices of
// 1024 rows with 16 rows per thread (the scans' cost spread over more rows;
// 8 groups for two passes, 7 for the single pass's three buffers a group),
// then 1024 and 2048 rows with 8 and 16 rows per thread
#define PFB_LGK(KL, KU, SV)                                                                                 \
    PFB_LG(16, 2, 8, KL, KU, SV), PFB_LG(16, 2, 7, KL, KU, SV), PFB_LG(8, 4, 4, KL, KU, SV),                 \
        PFB_LG(16, 4, 2, KL, KU, SV)

static const LongVariant kLongVariants[] = {
    PFB_LGK(0, 0, SV_TRI),   PFB_LGK(0, 1, SV_LOWER), PFB_LGK(0, 1, SV_NONE), PFB_LGK(0, 0, SV_LOWER),
    PFB_LGK(1, 0, SV_UPPER), PFB_LGK(1, 0, SV_NONE),  PFB_LGK(0, 0, SV_UPPER),
};

const LongVariant* find_long_variant(int shape, int KL, int KU, int SV)
{
    int n = 0;
    for (const LongVariant& v : kLongVariants)
        if (v.KL == KL && v.KU == KU && v.SV == SV && n++ == shape) return &v;
    return nullptr;
}

PFB_STREAM_STATUS_ACCESSOR(long_status_fetch_clear)

}  // namespace pfb
