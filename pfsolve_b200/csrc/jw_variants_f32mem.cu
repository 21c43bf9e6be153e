// jw_variants_f32mem.cu -- group-kernel variants, FP64 arithmetic on FP32 storage (doublePrecisionFloatMemory).
#include "jw_variant_defs.h"

namespace pfb {

static const JwVariant kPart[] = {
    PFB_F32_KINDS(PREC_F64_F32MEM),
};

const JwVariant* jw_variants_f32mem(int* count)
{
    *count = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace pfb
