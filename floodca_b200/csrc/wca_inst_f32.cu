// Step-kernel variants with FP32 state and FP64 accumulation (FCAB_PREC_F32),
// in both math modes.
#include "wca_dispatch.h"

namespace fcab {

bool lookup_f32(const VariantKey &k, Launchers *out)
{
    if (k.math == MATH_FAST)
        return lookup_kcr<float, double, MATH_FAST>(k, out);
    return lookup_kcr<float, double, MATH_EXACT>(k, out);
}

}  // namespace fcab
