// stream_variants_f64.cu -- streaming kernel variants, FP64.
#include "stream_variant_defs.h"

namespace pfb {

static const StreamVariant kPart[] = {
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

const StreamVariant* stream_variants_f64(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

PFB_STREAM_STATUS_ACCESSOR(stream_status_f64)

}  // namespace pfb
