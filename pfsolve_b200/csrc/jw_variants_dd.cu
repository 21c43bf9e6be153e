// jw_variants_dd.cu -- kernel variants: double-double.
#include "jw_variant_defs.h"

namespace pfb {

static const JwVariant kPart[] = {
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

const JwVariant* jw_variants_dd(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace pfb
