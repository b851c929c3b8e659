// eri_hm_0.cu -- Hermite-matrix ERI kernels with row pairs of Hermite level 0.
#include "eri_hermite.cuh"

namespace gci {
void register_hm_0(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]) { register_hm_row<0>(tab); }
} // namespace gci
