// Step-kernel variants with FP32 state and FP32 accumulation
// (FCAB_PREC_F32_ALL, the precision study's all-float run).
#include "wca_dispatch.h"

namespace fcab {

bool lookup_f32all(const VariantKey &k, Launchers *out)
{
    if (k.math != MATH_EXACT)
        return false;
    return lookup_kcr<float, float, MATH_EXACT>(k, out);
}

}  // namespace fcab
