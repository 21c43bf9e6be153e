// jw_variants_real.cu -- kernel variants: drop-in real JW and dgbmv applications.
#include "jw_variant_defs.h"

namespace pfb {

static const JwVariant kPart[] = {
    // JW application, real systems in place (upperBanded 2: tridiagonal;
    // 1: upper V / lower M; 0: lower V / upper M), by jw_type % 10.
    PFB_R4(0, 0, SV_TRI, LAY_REAL, LAY_REAL, false),    // ub 2, jwt 3
    PFB_R4(0, 1, SV_LOWER, LAY_REAL, LAY_REAL, false),  // ub 1, jwt 0
    PFB_R4(0, 1, SV_NONE, LAY_REAL, LAY_REAL, false),   // ub 1, jwt 1
    PFB_R4(0, 0, SV_LOWER, LAY_REAL, LAY_REAL, false),  // ub 1, jwt 2 / 3
    PFB_R4(1, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),  // ub 0, jwt 0
    PFB_R4(1, 0, SV_NONE, LAY_REAL, LAY_REAL, false),   // ub 0, jwt 1
    PFB_R4(0, 0, SV_UPPER, LAY_REAL, LAY_REAL, false),  // ub 0, jwt 2 / 3
    // dgbmv application (band matvec only), KL, KU <= 2
    PFB_R2(1, 1, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(2, 2, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(0, 2, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(2, 0, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(1, 2, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(2, 1, SV_NONE, LAY_REAL, LAY_REAL, false),
    PFB_R2(0, 0, SV_NONE, LAY_REAL, LAY_REAL, false),
};

const JwVariant* jw_variants_real(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace pfb
