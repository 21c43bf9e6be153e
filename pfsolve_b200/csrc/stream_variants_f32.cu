// stream_variants_f32.cu -- streaming kernel variants, FP32 storage and arithmetic (the reference's default precision).
#include "stream_variant_defs.h"

namespace pfb {

static const StreamVariant kPart[] = {
    // JW application on real systems
    PFB_SREALP(0, 0, SV_TRI, PREC_F32),
    PFB_SREALP(0, 1, SV_LOWER, PREC_F32),
    PFB_SREALP(0, 1, SV_NONE, PREC_F32),
    PFB_SREALP(0, 0, SV_LOWER, PREC_F32),
    PFB_SREALP(1, 0, SV_UPPER, PREC_F32),
    PFB_SREALP(1, 0, SV_NONE, PREC_F32),
    PFB_SREALP(0, 0, SV_UPPER, PREC_F32),
    // fused chains
    PFB_SREALP(1, 1, SV_UPPER, PREC_F32),
    PFB_SREALP(2, 2, SV_TRI, PREC_F32),
    PFB_SCPLXP(2, 2, SV_TRI, false, PREC_F32),
    PFB_SCPLXP(2, 2, SV_TRI, true, PREC_F32),
    PFB_SCPLXP(1, 1, SV_UPPER, true, PREC_F32),
};

const StreamVariant* stream_variants_f32(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

PFB_STREAM_STATUS_ACCESSOR(stream_status_f32)

}  // namespace pfb
