// eri_hm_3.cu -- Hermite-matrix ERI kernels with row pairs of Hermite level 3.
#include "eri_hermite.cuh"

namespace gci {
void register_hm_3(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]) { register_hm_row<3>(tab); }
} // namespace gci
