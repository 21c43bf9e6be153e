// jw_variants_chain.cu -- kernel variants: fused dgbmv -> JW -> block chains.
#include "jw_variant_defs.h"

namespace pfb {

static const JwVariant kPart[] = {
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
};

const JwVariant* jw_variants_chain(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace pfb
