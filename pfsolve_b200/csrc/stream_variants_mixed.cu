// stream_variants_mixed.cu -- streaming kernel variants, FP32 solve with FP64
// residual refinement (FP64 storage).
#include "stream_variant_defs.h"

namespace pfb {

static const StreamVariant kPart[] = {
    PFB_SREALP(0, 0, SV_TRI, PREC_MIXED),
    PFB_SREALP(0, 1, SV_LOWER, PREC_MIXED),
    PFB_SREALP(0, 0, SV_LOWER, PREC_MIXED),
    PFB_SREALP(1, 0, SV_UPPER, PREC_MIXED),
    PFB_SREALP(0, 0, SV_UPPER, PREC_MIXED),
    PFB_SREALP(1, 1, SV_UPPER, PREC_MIXED),
    PFB_SCPLXP(2, 2, SV_TRI, false, PREC_MIXED),
};

const StreamVariant* stream_variants_mixed(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

PFB_STREAM_STATUS_ACCESSOR(stream_status_mixed)

}  // namespace pfb
