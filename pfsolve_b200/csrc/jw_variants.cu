// jw_variants.cu -- explicit instantiations of the JW-step kernel and the
// standalone block / generic dgbmv kernels.
#include <vector>

#include "dd_kernel.cuh"
#include "jw_kernel.cuh"
#include "jw_variants.h"

namespace pfb {

template <class C>
static size_t smem_fn(int W, int G)
{
    return jw_smem_bytes<C>(W, G);
}

template <class C>
static void launch_fn(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const JwOperator& op, const JwIO& io, int W)
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
static size_t dd_smem_fn(int W, int G)
{
    return dd_smem_bytes<C>(W, G);
}
template <class C>
static void dd_launch_fn(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const JwOperator& op, const JwIO& io,
                         int W)
{
    jw_dd_kernel<C><<<grid, block, smem, st>>>(op, io, W);
}
#define PFB_DDV(R, KL, KU, SV, MEM)                                                                     \
    JwVariant{R, KL, KU, SV, LAY_REAL, LAY_REAL, 0, (MEM) ? 2 : 3, 0, 256,                              \
              (const void*)&jw_dd_kernel<DdCfg<R, KL, KU, SV, MEM>>, &dd_smem_fn<DdCfg<R, KL, KU, SV, MEM>>, \
              &dd_launch_fn<DdCfg<R, KL, KU, SV, MEM>>}
#define PFB_DD(KL, KU, SV) \
    PFB_DDV(4, KL, KU, SV, true), PFB_DDV(8, KL, KU, SV, true), PFB_DDV(4, KL, KU, SV, false), \
        PFB_DDV(8, KL, KU, SV, false)

// Rows-per-thread choices for the single-application (drop-in) variants.
#define PFB_R4(KL, KU, SV, LIN, LOUT, SC) \
    PFB_V(2, KL, KU, SV, LIN, LOUT, SC), PFB_V(4, KL, KU, SV, LIN, LOUT, SC), PFB_V(8, KL, KU, SV, LIN, LOUT, SC), \
        PFB_V(16, KL, KU, SV, LIN, LOUT, SC)
#define PFB_R2(KL, KU, SV, LIN, LOUT, SC) PFB_V(4, KL, KU, SV, LIN, LOUT, SC), PFB_V(8, KL, KU, SV, LIN, LOUT, SC)
#define PFB_M2(KL, KU, SV, LIN, LOUT, SC) \
    PFB_VP(4, KL, KU, SV, LIN, LOUT, SC, PREC_MIXED), PFB_VP(8, KL, KU, SV, LIN, LOUT, SC, PREC_MIXED)

static const JwVariant kVariants[] = {
    // JW application, real systems in place (upperBanded 2: tridiagonal;
    // 1: upper V / lower M; 0: lower V / upper M), by jw_type % 10.
    PFB_R4(0, 0, SV_TRI, LAY_REAL, LAY_REAL, false),    // ub 2, jwt 3
    PFB_R4(0, 1, SV_LOWER, LAY_REAL, LAY_REAL, false),  // ub 1, jwt 0
    PFB_R4(0, 1, SV_NONE, LAY_REAL, LAY_REAL, false),   // ub 1, jwt 1
    PFB_R4(0, 0, SV_LOWER, LAY_REAL, LAY_REAL, false),  // ub 1, jwt 2 / 3
    PFB_R4(1, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),  // ub 0, jwt 0
    PFB_R4(1, 0, SV_NONE, LAY_REAL, LAY_REAL, false),   // ub 0, jwt 1
    PFB_R4(0, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),  // ub 0, jwt 2 / 3
    // dgbmv application (band matvec only), KL, KU <= 2
    PFB_R2(1, 1, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(2, 2, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(0, 2, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(2, 0, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(1, 2, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(2, 1, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(0, 0, SV_NONE, LAY_REAL, LAY_REAL, false),
    // fused chains: dgbmv -> JW (-> block), real
    PFB_R2(1, 1, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_R2(1, 1, SV_LOWER, LAY_REAL, LAY_REAL, false),
    PFB_R2(1, 1, SV_TRI, LAY_REAL, LAY_REAL, false),
    PFB_R2(2, 2, SV_TRI, LAY_REAL, LAY_REAL, false),
    PFB_R2(0, 0, SV_TRI, LAY_REAL, LAY_REAL, true),
    PFB_R2(1, 1, SV_UPPER, LAY_REAL, LAY_REAL, true),
    // fused chains on complex XXII right-hand sides -> packed complex output
    PFB_R2(2, 2, SV_TRI, LAY_XXII, LAY_PACKED, false),
    PFB_R2(2, 2, SV_TRI, LAY_XXII, LAY_PACKED, true),
    PFB_R2(0, 0, SV_TRI, LAY_XXII, LAY_PACKED, false),
    PFB_R2(1, 1, SV_UPPER, LAY_XXII, LAY_PACKED, true),
    PFB_R2(1, 1, SV_UPPER, LAY_XXII, LAY_PACKED, false),
    PFB_R2(0, 0, SV_UPPER, LAY_XXII, LAY_PACKED, true),
    // mixed precision (FP32 solve + FP64 refinement), real
    PFB_M2(0, 0, SV_TRI, LAY_REAL, LAY_REAL, false),
    PFB_M2(0, 1, SV_LOWER, LAY_REAL, LAY_REAL, false),
    PFB_M2(0, 0, SV_LOWER, LAY_REAL, LAY_REAL, false),
    PFB_M2(1, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_M2(0, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_M2(1, 1, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_M2(2, 2, SV_TRI, LAY_XXII, LAY_PACKED, false),
    // coefficient-table variants for the single-matrix launches
    PFB_T2(0, 0, SV_TRI, LAY_REAL, LAY_REAL, false),
    PFB_T2(0, 1, SV_LOWER, LAY_REAL, LAY_REAL, false),
    PFB_T2(0, 0, SV_LOWER, LAY_REAL, LAY_REAL, false),
    PFB_T2(1, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_T2(0, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_T2(1, 1, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_T2(2, 2, SV_TRI, LAY_XXII, LAY_PACKED, false),
    PFB_T2(2, 2, SV_TRI, LAY_XXII, LAY_PACKED, true),
    PFB_T2(1, 1, SV_UPPER, LAY_XXII, LAY_PACKED, true),
    // double-double (quad emulation), real systems
    PFB_DD(0, 0, SV_TRI),
    PFB_DD(0, 1, SV_LOWER),
    PFB_DD(0, 1, SV_NONE),
    PFB_DD(0, 0, SV_LOWER),
    PFB_DD(1, 0, SV_UPPER),
    PFB_DD(1, 0, SV_NONE),
    PFB_DD(0, 0, SV_UPPER),
    PFB_DD(1, 1, SV_UPPER),
    PFB_DD(1, 1, SV_NONE),
};

const JwVariant* find_jw_variant(int R, int KL, int KU, int SV, int LIN, int LOUT, int SCALE, int PREC, int TBL)
{
    for (const JwVariant& v : kVariants)
        if (v.R == R && v.KL == KL && v.KU == KU && v.SV == SV && v.LIN == LIN && v.LOUT == LOUT &&
            v.SCALE == (SCALE ? 1 : 0) && v.PREC == PREC && v.TBL == (TBL ? 1 : 0))
            return &v;
    return nullptr;
}

const JwVariant* jw_variants(int* count)
{
    *count = (int)(sizeof(kVariants) / sizeof(kVariants[0]));
    return kVariants;
}

// ---------------------------------------------------------------------------
// Block application: element (x, y) of a size0 x size1 array
// (PfSolve/pfSolve_CodeGen/pfSolve_KernelsLevel2/pfSolve_block.h:37-115).
// HBM-bound elementwise work: a grid-stride loop over rows y with the threads
// of a block striding x, so reads and writes of each row are coalesced.
__global__ void __launch_bounds__(256) block_kernel(const BlockArgs a)
{
    const int bt = a.layout;
    for (int64_t y = blockIdx.x; y < a.size1; y += gridDim.x) {
        const int64_t ii = a.in_off + y * a.in_stride;
        const int64_t oi = a.out_off + y * a.out_stride;
        for (int64_t x = threadIdx.x; x < a.size0; x += blockDim.x) {
            double vr = 0.0, vi = 0.0;
            if (!a.skip_read) {
                if (x >= a.iz0 && x < a.iz1) {
                    switch (bt) {
                    case 1: vr = a.in[ii + x]; break;
                    case 2: case 3: case 4: {
                        const double2 v = reinterpret_cast<const double2*>(a.in)[ii + x];
                        vr = v.x;
                        vi = v.y;
                        break;
                    }
                    case 5: vr = a.in[ii + x]; break;
                    case 6: vi = a.in[ii + x]; break;
                    default: vr = a.in[2 * ii + x]; vi = a.in[2 * ii + x + a.in_stride]; break;
                    }
                }
                if (a.scale_kind) {
                    const double f = scale_factor(a.scale_kind, x, a.lshift, a.s);
                    vr *= f;
                    vi *= f;
                }
            }
            if (x < a.oz0 || x >= a.oz1) continue;
            switch (bt) {
            case 1: case 2: {
                double* p = a.out + oi + x;
                *p = a.accumulate ? vr + *p : vr;
                break;
            }
            case 3: {
                double* p = a.out + oi + x;
                *p = a.accumulate ? vi + *p : vi;
                break;
            }
            case 4:
                a.out[2 * oi + x] = vr;
                a.out[2 * oi + x + a.out_stride] = vi;
                break;
            default: {
                double2* p = reinterpret_cast<double2*>(a.out) + oi + x;
                if (a.accumulate) {
                    const double2 o = *p;
                    vr += o.x;
                    vi += o.y;
                }
                *p = make_double2(vr, vi);
                break;
            }
            }
        }
    }
}

void launch_block(const BlockArgs& a, cudaStream_t st, int num_sms)
{
    int64_t blocks = a.size1;
    const int64_t cap = (int64_t)num_sms * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    block_kernel<<<(unsigned)blocks, 256, 0, st>>>(a);
}

// ---------------------------------------------------------------------------
// dgbmv with any bandwidth (pfSolve_KernelsLevel1/pfSolve_MatVecMul.h:383-446):
// one block per system, the system staged in shared memory (zero outside the
// input keep-window), y_r = sum_j A[off + j*M + c] x_c, c = r + ku - j.
__global__ void __launch_bounds__(256) dgbmv_generic_kernel(const DgbmvArgs a)
{
    extern __shared__ double xs[];
    for (int64_t sys = blockIdx.x; sys < a.nsys; sys += gridDim.x) {
        double* x = a.x + a.off_x + sys * a.stride;
        for (int64_t r = threadIdx.x; r < a.M; r += blockDim.x)
            xs[r] = (r >= a.iz0 && r < a.iz1) ? x[r] : 0.0;
        __syncthreads();
        for (int64_t r = threadIdx.x; r < a.M; r += blockDim.x) {
            double acc = 0.0;
            for (int j = 0; j < a.lda; ++j) {
                const int64_t c = r + a.ku - j;
                if (c < 0 || c >= a.M) continue;
                acc = __fma_rn(__ldg(a.A + a.off_A + (int64_t)j * a.M + c), xs[c], acc);
            }
            if (r >= a.oz0 && r < a.oz1) x[r] = acc;
        }
        __syncthreads();
    }
}

void launch_dgbmv_generic(const DgbmvArgs& a, cudaStream_t st, int num_sms)
{
    int64_t blocks = a.nsys;
    const int64_t cap = (int64_t)num_sms * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    const size_t smem = (size_t)a.M * sizeof(double);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(dgbmv_generic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dgbmv_generic_kernel<<<(unsigned)blocks, 256, smem, st>>>(a);
}

}  // namespace pfb
