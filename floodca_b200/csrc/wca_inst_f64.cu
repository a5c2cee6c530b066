// Step-kernel variants in FP64 (FCAB_PREC_F64, the reference's FCA_DOUBLE
// build and the precision study's oracle run).
#include "wca_dispatch.h"

namespace fcab {

bool lookup_f64(const VariantKey &k, Launchers *out)
{
    return lookup_kcr<double, double, MATH_EXACT>(k, out);
}

}  // namespace fcab
