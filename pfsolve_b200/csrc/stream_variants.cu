// stream_variants.cu -- lookup over the streaming kernel variant tables
// (stream_variants_*.cu), the TMA tensor maps that describe a launch's
// right-hand sides, and the status of the kernels' bounded waits.
#include <cuda.h>

#include <algorithm>

#include "jw_variants.h"

namespace pfb {

const StreamVariant* stream_variants_f64(int* count);
const StreamVariant* stream_variants_mixed(int* count);
const StreamVariant* stream_variants_alt(int* count);
const StreamVariant* stream_variants_f32(int* count);
const StreamVariant* stream_variants_f32mem(int* count);
unsigned stream_status_f64();
unsigned stream_status_mixed();
unsigned stream_status_alt();
unsigned stream_status_f32();
unsigned stream_status_f32mem();

const StreamVariant* find_stream_variant(int R, int W, int KL, int KU, int SV, int LIN, int LOUT, int SCALE, int PREC,
                                         int ALT)
{
    for (auto part : {stream_variants_f64, stream_variants_mixed, stream_variants_alt, stream_variants_f32,
                      stream_variants_f32mem}) {
        int n = 0;
        const StreamVariant* vs = part(&n);
        for (int i = 0; i < n; ++i) {
            const StreamVariant& v = vs[i];
            if (v.R == R && v.W == W && v.KL == KL && v.KU == KU && v.SV == SV && v.LIN == LIN && v.LOUT == LOUT &&
                v.SCALE == (SCALE ? 1 : 0) && v.PREC == PREC && v.ALT == (ALT ? 1 : 0))
                return &v;
        }
    }
    return nullptr;
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

// 3-D view of a set of rows of `es`-byte elements (FP64 or FP32): {row in
// chunk (inner, `inner` elements), chunk (`chunks`, `inner` elements apart),
// row set (`sets`, `set_stride` bytes apart)}; box {box_units 16-byte units,
// 32 chunks, 1 set}.
bool encode_rows(CUtensorMap* map, const void* base, int64_t inner, int64_t chunks, int64_t sets, int64_t set_stride,
                 int box_units, int es)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn || (es != 4 && es != 8)) return false;
    if (reinterpret_cast<uintptr_t>(base) % 16 || set_stride % 16 || set_stride <= 0 || sets < 1 || sets > INT32_MAX ||
        (inner * es) % 16)
        return false;
    const cuuint64_t dims[3] = {(cuuint64_t)inner, (cuuint64_t)chunks, (cuuint64_t)sets};
    const cuuint64_t strides[2] = {(cuuint64_t)(inner * es), (cuuint64_t)set_stride};
    const cuuint32_t box[3] = {(cuuint32_t)(box_units * (16 / es)), 32u, 1u};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    return fn(map, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
              const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(box_units), CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

bool encode_row_maps(int R_, int LIN, int LOUT, int IB, int IBO, const JwIO& io, CUtensorMap* in, CUtensorMap* out,
                     int es)
{
    const int64_t R = R_, M = io.M;
    if (M % R != 0 || io.nsys < 1) return false;
    const int64_t chunks = M / R;
    const bool cplx = LIN != LAY_REAL;
    const int64_t sets = cplx ? 2 * io.nsys : io.nsys;
    const char* in0 = reinterpret_cast<const char*>(io.in) + io.in_off * es;
    char* out0 = reinterpret_cast<char*>(io.out);
    if (!encode_rows(in, in0, R, chunks, sets, io.in_stride * es, IB, es)) return false;
    if (LOUT == LAY_PACKED)  // complex elements of 2 es bytes: 2 R storage elements per chunk
        return encode_rows(out, out0 + io.out_off * 2 * es, 2 * R, chunks, io.nsys, io.out_stride * 2 * es, IBO, es);
    const int64_t osets = (LOUT == LAY_XXII) ? 2 * io.nsys : io.nsys;
    return encode_rows(out, out0 + io.out_off * es, R, chunks, osets, io.out_stride * es, IBO, es);
}

bool encode_seq_maps(const JwIO& io, int64_t M_in, int64_t M_out, int CH, CUtensorMap* in, CUtensorMap* out)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn || io.nsys < 1 || io.nsys > INT32_MAX || M_in < 1 || M_out < 1) return false;
    if (io.in != io.out || io.in_off != io.out_off || io.in_stride != io.out_stride) return false;
    const double* base = io.in + io.in_off;
    const int64_t stride = io.in_stride * 8;
    if (reinterpret_cast<uintptr_t>(base) % 16 || stride % 16 || io.in_stride < std::max(M_in, M_out)) return false;
    const cuuint64_t strides[1] = {(cuuint64_t)stride};
    if (CH != 8 && CH != 16) return false;
    const cuuint32_t box[2] = {(cuuint32_t)CH, 32u};
    const cuuint32_t estr[2] = {1u, 1u};
    const cuuint64_t din[2] = {(cuuint64_t)M_in, (cuuint64_t)io.nsys};
    const cuuint64_t dout[2] = {(cuuint64_t)M_out, (cuuint64_t)io.nsys};
    const CUtensorMapSwizzle swz = CH == 16 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
    return fn(in, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), din, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
           fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dout, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool encode_batch_seq_maps(const JwIO& io, BatchSeqEntry* e)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn || io.nsys < 1 || io.nsys > INT32_MAX || io.M < 1 || io.out_stride < io.M) return false;
    const cuuint32_t estr[2] = {1u, 1u};
    // output: packed complex rows, 16 bytes each; the map ends at 2 M doubles
    double* obase = io.out + 2 * io.out_off;
    if (reinterpret_cast<uintptr_t>(obase) % 16) return false;
    const cuuint64_t ostr[1] = {(cuuint64_t)io.out_stride * 16};
    const cuuint64_t dout[2] = {(cuuint64_t)(2 * io.M), (cuuint64_t)io.nsys};
    const cuuint32_t bout[2] = {16u, 32u};
    if (fn(&e->out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, obase, dout, ostr, bout, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    // input: a system's real rows then its imaginary rows, one tensor row
    e->tma_in = 0;
    const double* ibase = io.in + io.in_off;
    if (reinterpret_cast<uintptr_t>(ibase) % 16 == 0 && io.in_stride >= io.M && 2 * io.in_stride <= INT32_MAX) {
        const cuuint64_t istr[1] = {(cuuint64_t)io.in_stride * 16};
        const cuuint64_t din[2] = {(cuuint64_t)(2 * io.in_stride), (cuuint64_t)io.nsys};
        const cuuint32_t b8[2] = {8u, 32u}, b16[2] = {16u, 32u};
        e->tma_in = fn(&e->in[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(ibase), din, istr, b8, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
                    fn(&e->in[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(ibase), din, istr, b16, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    return true;
}

bool encode_stream_maps(const StreamVariant* v, const JwIO& io, CUtensorMap* in, CUtensorMap* out)
{
    return encode_row_maps(v->R, v->LIN, v->LOUT, v->IB, v->IBO, io, in, out, prec_f32_storage(v->PREC) ? 4 : 8);
}

unsigned stream_status_fetch_clear()
{
    const unsigned a = stream_status_f64(), b = stream_status_mixed(), c = cluster_status_fetch_clear();
    const unsigned d = steps_status_fetch_clear(), e = batch_status_fetch_clear(), f = long_status_fetch_clear();
    const unsigned g = stream_status_alt(), h = stream_status_f32(), i = stream_status_f32mem();
    if (a == ~0u || b == ~0u || c == ~0u || d == ~0u || e == ~0u || f == ~0u || g == ~0u || h == ~0u || i == ~0u)
        return ~0u;
    return a | b | c | d | e | f | g | h | i;
}

}  // namespace pfb
