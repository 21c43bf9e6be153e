// stream_variants_alt.cu -- streaming kernel variants for ALT stride-2 mode
// (FP64, real row sets of two systems each; the operator kinds of the real
// table in stream_variants_f64.cu with a one-row band halo).
#include "stream_variant_defs.h"

namespace pfb {

static const StreamVariant kPart[] = {
    PFB_SALT(0, 0, SV_TRI),
    PFB_SALT(0, 1, SV_LOWER),
    PFB_SALT(0, 1, SV_NONE),
    PFB_SALT(0, 0, SV_LOWER),
    PFB_SALT(1, 0, SV_UPPER),
    PFB_SALT(1, 0, SV_NONE),
    PFB_SALT(0, 0, SV_UPPER),
};

const StreamVariant* stream_variants_alt(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

PFB_STREAM_STATUS_ACCESSOR(stream_status_alt)

}  // namespace pfb
