// Batched-ensemble step-kernel variants (FP32 state, FP64 accumulation).
#include "wca_dispatch.h"

namespace fcab {

template <int MATH>
static bool lookup_batch_math(const VariantKey &k, BatchLaunchers *out)
{
#define FCAB_BCASE(KK, CC, RR)                                                           \
    if (k.K == KK && k.cpl == CC && (k.rainf != 0) == RR) {                              \
        if (k.landonly) {                                                                \
            out->step = &launch_batch<float, double, KK, CC, MATH, RR, true>;            \
            out->step_fn = (const void *)&k_step_batch<float, double, KK, CC, MATH, RR, true>; \
        } else {                                                                         \
            out->step = &launch_batch<float, double, KK, CC, MATH, RR, false>;           \
            out->step_fn = (const void *)&k_step_batch<float, double, KK, CC, MATH, RR, false>; \
        }                                                                                \
        out->window = &launch_window<float>;                                             \
        out->vfull = &launch_batch_vfull<float, KK, MATH>;                               \
        return true;                                                                     \
    }
    FCAB_BCASE(4, 1, false) FCAB_BCASE(4, 1, true)
    FCAB_BCASE(4, 2, false) FCAB_BCASE(4, 2, true)
    FCAB_BCASE(4, 4, false) FCAB_BCASE(4, 4, true)
    FCAB_BCASE(8, 1, false) FCAB_BCASE(8, 1, true)
    FCAB_BCASE(8, 2, false) FCAB_BCASE(8, 2, true)
#undef FCAB_BCASE
    return false;
}

bool lookup_batch_f32(const VariantKey &k, BatchLaunchers *out)
{
    if (k.prec != 0)
        return false;
    return k.math == MATH_FAST ? lookup_batch_math<MATH_FAST>(k, out)
                               : lookup_batch_math<MATH_EXACT>(k, out);
}

}  // namespace fcab
