// stream_variants.cu -- instantiations of the streaming JW-step kernel, the
// TMA tensor maps that describe a launch's right-hand sides, and the device
// status word of its bounded waits.
#include <cuda.h>

#include "jw_stream.cuh"
#include "jw_variants.h"

namespace pfb {

template <class C>
static size_t st_smem_fn(int G)
{
    return st_smem_bytes<C>(G);
}

template <class C>
static void st_launch_fn(dim3 grid, dim3 block, size_t smem, cudaStream_t st, const CUtensorMap* in,
                         const CUtensorMap* out, const JwOperator& op, const JwIO& io)
{
    jw_stream_kernel<C><<<grid, block, smem, st>>>(*in, *out, op, io);
}

#define PFB_SV(R, W, KL, KU, SV, LIN, LOUT, SC)                                                               \
    StreamVariant{R, W, KL, KU, SV, LIN, LOUT, SC, StCfg<R, W, KL, KU, SV, LIN, LOUT, SC>::kMaxThreads,          \
                  (const void*)&jw_stream_kernel<StCfg<R, W, KL, KU, SV, LIN, LOUT, SC>>,                        \
                  &st_smem_fn<StCfg<R, W, KL, KU, SV, LIN, LOUT, SC>>, StCfg<R, W, KL, KU, SV, LIN, LOUT, SC>::IB, \
                  StCfg<R, W, KL, KU, SV, LIN, LOUT, SC>::IBO, &st_launch_fn<StCfg<R, W, KL, KU, SV, LIN, LOUT, SC>>}
// real systems: 8 rows per thread (M <= 256, 512, 1024), 16 (M <= 512, 1024,
// 2048) and 32 (M <= 1024, 2048, 4096)
#define PFB_SREAL(KL, KU, SV)                                                                                   \
    PFB_SV(8, 1, KL, KU, SV, LAY_REAL, LAY_REAL, false), PFB_SV(8, 2, KL, KU, SV, LAY_REAL, LAY_REAL, false),   \
        PFB_SV(8, 4, KL, KU, SV, LAY_REAL, LAY_REAL, false), PFB_SV(16, 1, KL, KU, SV, LAY_REAL, LAY_REAL, false), \
        PFB_SV(16, 2, KL, KU, SV, LAY_REAL, LAY_REAL, false), PFB_SV(16, 4, KL, KU, SV, LAY_REAL, LAY_REAL, false), \
        PFB_SV(32, 1, KL, KU, SV, LAY_REAL, LAY_REAL, false), PFB_SV(32, 2, KL, KU, SV, LAY_REAL, LAY_REAL, false), \
        PFB_SV(32, 4, KL, KU, SV, LAY_REAL, LAY_REAL, false)
// complex XXII right-hand sides written packed
#define PFB_SCPLX(KL, KU, SV, SC)                                                                           \
    PFB_SV(16, 1, KL, KU, SV, LAY_XXII, LAY_PACKED, SC), PFB_SV(16, 2, KL, KU, SV, LAY_XXII, LAY_PACKED, SC), \
        PFB_SV(32, 1, KL, KU, SV, LAY_XXII, LAY_PACKED, SC), PFB_SV(32, 2, KL, KU, SV, LAY_XXII, LAY_PACKED, SC)

static const StreamVariant kStreamVariants[] = {
    // JW application on real systems (see kVariants for the operator kinds)
    PFB_SREAL(0, 0, SV_TRI),
    PFB_SREAL(0, 1, SV_LOWER),
    PFB_SREAL(0, 1, SV_NONE),
    PFB_SREAL(0, 0, SV_LOWER),
    PFB_SREAL(1, 0, SV_UPPER),
    PFB_SREAL(1, 0, SV_NONE),
    PFB_SREAL(0, 0, SV_UPPER),
    // fused chains
    PFB_SREAL(1, 1, SV_UPPER),
    PFB_SREAL(2, 2, SV_TRI),
    PFB_SCPLX(2, 2, SV_TRI, false),
    PFB_SCPLX(2, 2, SV_TRI, true),
    PFB_SCPLX(1, 1, SV_UPPER, true),
};

const StreamVariant* find_stream_variant(int R, int W, int KL, int KU, int SV, int LIN, int LOUT, int SCALE)
{
    for (const StreamVariant& v : kStreamVariants)
        if (v.R == R && v.W == W && v.KL == KL && v.KU == KU && v.SV == SV && v.LIN == LIN && v.LOUT == LOUT &&
            v.SCALE == (SCALE ? 1 : 0))
            return &v;
    return nullptr;
}

const StreamVariant* stream_variants(int* count)
{
    *count = (int)(sizeof(kStreamVariants) / sizeof(kStreamVariants[0]));
    return kStreamVariants;
}

// ---- Tensor maps.  cuTensorMapEncodeTiled is a host-side driver entry
// point, resolved once through the runtime.
namespace {
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiledFn) nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

CUtensorMapSwizzle swizzle_for(int units)
{
    switch (units) {
    case 8: return CU_TENSOR_MAP_SWIZZLE_128B;
    case 4: return CU_TENSOR_MAP_SWIZZLE_64B;
    case 2: return CU_TENSOR_MAP_SWIZZLE_32B;
    default: return CU_TENSOR_MAP_SWIZZLE_NONE;
    }
}

// 3-D view of a set of rows: {row in chunk (inner, `inner` doubles), chunk
// (`chunks`, `inner` doubles apart), row set (`sets`, `set_stride` bytes apart)};
// box {box_units * 2 doubles, 32 chunks, 1 set}.
bool encode_rows(CUtensorMap* map, const void* base, int64_t inner, int64_t chunks, int64_t sets, int64_t set_stride,
                 int box_units)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    if (reinterpret_cast<uintptr_t>(base) % 16 || set_stride % 16 || set_stride <= 0 || sets < 1 || sets > INT32_MAX)
        return false;
    const cuuint64_t dims[3] = {(cuuint64_t)inner, (cuuint64_t)chunks, (cuuint64_t)sets};
    const cuuint64_t strides[2] = {(cuuint64_t)(inner * 8), (cuuint64_t)set_stride};
    const cuuint32_t box[3] = {(cuuint32_t)(box_units * 2), 32u, 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(box_units), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

bool encode_stream_maps(const StreamVariant* v, const JwIO& io, CUtensorMap* in, CUtensorMap* out)
{
    const int64_t R = v->R, M = io.M;
    if (M % R != 0 || io.nsys < 1) return false;
    const int64_t chunks = M / R;
    const bool cplx = v->LIN != LAY_REAL;
    const int64_t sets = cplx ? 2 * io.nsys : io.nsys;
    if (!encode_rows(in, io.in + io.in_off, R, chunks, sets, io.in_stride * 8, v->IB)) return false;
    if (v->LOUT == LAY_PACKED)
        return encode_rows(out, reinterpret_cast<const double2*>(io.out) + io.out_off, 2 * R, chunks, io.nsys,
                           io.out_stride * 16, v->IBO);
    const int64_t osets = (v->LOUT == LAY_XXII) ? 2 * io.nsys : io.nsys;
    return encode_rows(out, io.out + io.out_off, R, chunks, osets, io.out_stride * 8, v->IBO);
}

unsigned stream_status_fetch_clear()
{
    unsigned v = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&v, g_stream_status, sizeof(v)) != cudaSuccess) return ~0u;
    if (v) cudaMemcpyToSymbol(g_stream_status, &zero, sizeof(zero));
    return v;
}

}  // namespace pfb
