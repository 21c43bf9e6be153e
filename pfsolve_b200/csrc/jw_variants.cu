// jw_variants.cu -- lookup over the kernel variant tables (jw_variants_*.cu)
// and the standalone block / generic dgbmv kernels.
#include <vector>

#include "jw_kernel.cuh"
#include "jw_variants.h"
#include "plan.h"

namespace pfb {

const JwVariant* jw_variants_real(int* count);
const JwVariant* jw_variants_chain(int* count);
const JwVariant* jw_variants_mixed(int* count);
const JwVariant* jw_variants_dd(int* count);
const JwVariant* jw_variants_f32(int* count);
const JwVariant* jw_variants_f32mem(int* count);

namespace {
using PartFn = const JwVariant* (*)(int*);
const PartFn kParts[] = {jw_variants_real, jw_variants_chain, jw_variants_mixed, jw_variants_dd, jw_variants_f32,
                         jw_variants_f32mem};
}  // namespace

const JwVariant* find_jw_variant(int R, int KL, int KU, int SV, int LIN, int LOUT, int SCALE, int PREC, int TBL)
{
    for (PartFn part : kParts) {
        int n = 0;
        const JwVariant* vs = part(&n);
        for (int i = 0; i < n; ++i) {
            const JwVariant& v = vs[i];
            if (v.R == R && v.KL == KL && v.KU == KU && v.SV == SV && v.LIN == LIN && v.LOUT == LOUT &&
                v.SCALE == (SCALE ? 1 : 0) && v.PREC == PREC && v.TBL == (TBL ? 1 : 0))
                return &v;
        }
    }
    return nullptr;
}

// ---------------------------------------------------------------------------
// Block application: element (x, y) of a size0 x size1 array
// (PfSolve/pfSolve_CodeGen/pfSolve_KernelsLevel2/pfSolve_block.h:37-115).
// HBM-bound elementwise work: a grid-stride loop over rows y with the threads
// of a block striding x, so reads and writes of each row are coalesced.
// T: the storage type (FP64, or FP32 for the FP32-storage precisions); values
// are widened to FP64 in registers and rounded once on store.
template <class T>
__global__ void __launch_bounds__(256) block_kernel(const BlockArgs a)
{
    using T2 = typename Vec2Of<T>::type;
    const T* in = reinterpret_cast<const T*>(a.in);
    T* out = reinterpret_cast<T*>(a.out);
    const int bt = a.layout;
    for (int64_t y = blockIdx.x; y < a.size1; y += gridDim.x) {
        const int64_t ii = a.in_off + y * a.in_stride;
        const int64_t oi = a.out_off + y * a.out_stride;
        for (int64_t x = threadIdx.x; x < a.size0; x += blockDim.x) {
            double vr = 0.0, vi = 0.0;
            if (!a.skip_read) {
                if (x >= a.iz0 && x < a.iz1) {
                    switch (bt) {
                    case 1: vr = in[ii + x]; break;
                    case 2: case 3: case 4: {
                        const T2 v = reinterpret_cast<const T2*>(in)[ii + x];
                        vr = v.x;
                        vi = v.y;
                        break;
                    }
                    case 5: vr = in[ii + x]; break;
                    case 6: vi = in[ii + x]; break;
                    default: vr = in[2 * ii + x]; vi = in[2 * ii + x + a.in_stride]; break;
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
                T* p = out + oi + x;
                *p = (T)(a.accumulate ? vr + (double)*p : vr);
                break;
            }
            case 3: {
                T* p = out + oi + x;
                *p = (T)(a.accumulate ? vi + (double)*p : vi);
                break;
            }
            case 4:
                out[2 * oi + x] = (T)vr;
                out[2 * oi + x + a.out_stride] = (T)vi;
                break;
            default: {
                T2* p = reinterpret_cast<T2*>(out) + oi + x;
                if (a.accumulate) {
                    const T2 o = *p;
                    vr += o.x;
                    vi += o.y;
                }
                *p = T2{(T)vr, (T)vi};
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
    if (a.f32) block_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(a);
    else block_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(a);
}

// ---------------------------------------------------------------------------
// dgbmv with any bandwidth (pfSolve_KernelsLevel1/pfSolve_MatVecMul.h:383-446):
// one block per system, the system staged in shared memory (zero outside the
// input keep-window), y_r = sum_j A[off + j*M + c] x_c, c = r + ku - j.
// T: the storage type of A and x; the sums run in FP64.
template <class T>
__global__ void __launch_bounds__(256) dgbmv_generic_kernel(const DgbmvArgs a)
{
    extern __shared__ double xs[];
    const T* A = reinterpret_cast<const T*>(a.A);
    for (int64_t sys = blockIdx.x; sys < a.nsys; sys += gridDim.x) {
        T* x = reinterpret_cast<T*>(a.x) + a.off_x + sys * a.stride;
        for (int64_t r = threadIdx.x; r < a.M; r += blockDim.x)
            xs[r] = (r >= a.iz0 && r < a.iz1) ? (double)x[r] : 0.0;
        __syncthreads();
        for (int64_t r = threadIdx.x; r < a.M; r += blockDim.x) {
            double acc = 0.0;
            for (int j = 0; j < a.lda; ++j) {
                const int64_t c = r + a.ku - j;
                if (c < 0 || c >= a.M || (j < 64 && ((a.skip >> j) & 1))) continue;
                acc = __fma_rn((double)__ldg(A + a.off_A + (int64_t)j * a.M + c), xs[c], acc);
            }
            if (r >= a.oz0 && r < a.oz1) x[r] = (T)acc;
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
    if (a.f32) {
        if (smem > 48 * 1024) allow_max_smem((const void*)dgbmv_generic_kernel<float>);
        dgbmv_generic_kernel<float><<<(unsigned)blocks, 256, smem, st>>>(a);
    } else {
        if (smem > 48 * 1024) allow_max_smem((const void*)dgbmv_generic_kernel<double>);
        dgbmv_generic_kernel<double><<<(unsigned)blocks, 256, smem, st>>>(a);
    }
}

}  // namespace pfb
