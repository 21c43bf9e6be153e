// cluster_variants.cu -- instantiations of the long-system (cluster) JW-step
// kernel, their cluster launch, and the status word of their bounded waits.
#include <cuda.h>

#include "jw_cluster.cuh"
#include "jw_variants.h"
#include "stream_variant_defs.h"

namespace pfb {

template <class C>
static cudaError_t cl_launch_fn(int clusters, size_t smem, cudaStream_t st, const CUtensorMap* in,
                                const CUtensorMap* out, const JwOperator& op, const JwIO& io)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(clusters * C::C));
    cfg.blockDim = dim3((unsigned)C::T);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C::C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, jw_cluster_kernel<C>, *in, *out, op, io);
}

template <class C>
static int cl_max_clusters(size_t smem)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)C::C);
    cfg.blockDim = dim3((unsigned)C::T);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C::C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (const void*)jw_cluster_kernel<C>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

#define PFB_CL(R, W, CC, KL, KU, SV)                                                                          \
    ClusterVariant{R, W, CC, KL, KU, SV, (const void*)&jw_cluster_kernel<ClCfg<R, W, CC, KL, KU, SV>>,        \
                   cl_smem_bytes<ClCfg<R, W, CC, KL, KU, SV>>(), ClCfg<R, W, CC, KL, KU, SV>::B::IB,          \
                   ClCfg<R, W, CC, KL, KU, SV>::B::IBO, &cl_launch_fn<ClCfg<R, W, CC, KL, KU, SV>>,           \
                   &cl_max_clusters<ClCfg<R, W, CC, KL, KU, SV>>}
// slices of 2048 rows (8 warps x 32 threads x 8 rows): N <= 6144, 8192,
// 12288, 16384 with 3, 4, 6, 8 CTAs per cluster
#define PFB_CLK(KL, KU, SV) \
    PFB_CL(8, 8, 3, KL, KU, SV), PFB_CL(8, 8, 4, KL, KU, SV), PFB_CL(8, 8, 6, KL, KU, SV), PFB_CL(8, 8, 8, KL, KU, SV)

static const ClusterVariant kClusterVariants[] = {
    PFB_CLK(0, 0, SV_TRI),   PFB_CLK(0, 1, SV_LOWER), PFB_CLK(0, 1, SV_NONE), PFB_CLK(0, 0, SV_LOWER),
    PFB_CLK(1, 0, SV_UPPER), PFB_CLK(1, 0, SV_NONE),  PFB_CLK(0, 0, SV_UPPER),
};

const ClusterVariant* find_cluster_variant(int C, int KL, int KU, int SV)
{
    for (const ClusterVariant& v : kClusterVariants)
        if (v.C == C && v.KL == KL && v.KU == KU && v.SV == SV) return &v;
    return nullptr;
}

PFB_STREAM_STATUS_ACCESSOR(cluster_status_fetch_clear)

}  // namespace pfb
