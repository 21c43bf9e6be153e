// jw_variants_mixed.cu -- kernel variants: mixed precision and coefficient-table.
#include "jw_variant_defs.h"

namespace pfb {

static const JwVariant kPart[] = {
    // mixed precision (FP32 solve + FP64 refinement), real
    PFB_M2(0, 0, SV_TRI, LAY_REAL, LAY_REAL, false),
    PFB_M2(0, 1, SV_LOWER, LAY_REAL, LAY_REAL, false),
    PFB_M2(0, 0, SV_LOWER, LAY_REAL, LAY_REAL, false),
    PFB_M2(1, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_M2(0, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_M2(1, 1, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_M2(2, 2, SV_TRI, LAY_XXII, LAY_PACKED, false),
    // coefficient-table variants for the single-matrix launches
    PFB_T2(0, 0, SV_TRI, LAY_REAL, LAY_REAL, false),
    PFB_T2(0, 1, SV_LOWER, LAY_REAL, LAY_REAL, false),
    PFB_T2(0, 0, SV_LOWER, LAY_REAL, LAY_REAL, false),
    PFB_T2(1, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_T2(0, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_T2(1, 1, SV_UPPER, LAY_REAL, LAY_REAL, false),
    PFB_T2(2, 2, SV_TRI, LAY_XXII, LAY_PACKED, false),
    PFB_T2(2, 2, SV_TRI, LAY_XXII, LAY_PACKED, true),
    PFB_T2(1, 1, SV_UPPER, LAY_XXII, LAY_PACKED, true),
};

const JwVariant* jw_variants_mixed(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace pfb
