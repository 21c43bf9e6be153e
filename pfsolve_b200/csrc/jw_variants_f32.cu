// jw_variants_f32.cu -- group-kernel variants, FP32 storage and arithmetic (the reference's default precision).
#include "jw_variant_defs.h"

namespace pfb {

static const JwVariant kPart[] = {
    PFB_F32_KINDS(PREC_F32),
};

const JwVariant* jw_variants_f32(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace pfb
