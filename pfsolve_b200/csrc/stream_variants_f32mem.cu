// stream_variants_f32mem.cu -- streaming kernel variants, FP64 arithmetic on FP32 storage (doublePrecisionFloatMemory).
#include "stream_variant_defs.h"

namespace pfb {

static const StreamVariant kPart[] = {
    // JW application on real systems
    PFB_SREALP(0, 0, SV_TRI, PREC_F64_F32MEM),
    PFB_SREALP(0, 1, SV_LOWER, PREC_F64_F32MEM),
    PFB_SREALP(0, 1, SV_NONE, PREC_F64_F32MEM),
    PFB_SREALP(0, 0, SV_LOWER, PREC_F64_F32MEM),
    PFB_SREALP(1, 0, SV_UPPER, PREC_F64_F32MEM),
    PFB_SREALP(1, 0, SV_NONE, PREC_F64_F32MEM),
    PFB_SREALP(0, 0, SV_UPPER, PREC_F64_F32MEM),
    // fused chains
    PFB_SREALP(1, 1, SV_UPPER, PREC_F64_F32MEM),
    PFB_SREALP(2, 2, SV_TRI, PREC_F64_F32MEM),
    PFB_SCPLXP(2, 2, SV_TRI, false, PREC_F64_F32MEM),
    PFB_SCPLXP(2, 2, SV_TRI, true, PREC_F64_F32MEM),
    PFB_SCPLXP(1, 1, SV_UPPER, true, PREC_F64_F32MEM),
};

const StreamVariant* stream_variants_f32mem(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

PFB_STREAM_STATUS_ACCESSOR(stream_status_f32mem)

}  // namespace pfb
