// eri_hm_5.cu -- Hermite-matrix ERI kernels with row pairs of Hermite level 5.
#include "eri_hermite.cuh"

namespace gci {
void register_hm_5(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]) { register_hm_row<5>(tab); }
} // namespace gci
