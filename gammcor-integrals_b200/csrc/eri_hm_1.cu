// eri_hm_1.cu -- Hermite-matrix ERI kernels with row pairs of Hermite level 1.
#include "eri_hermite.cuh"

namespace gci {
void register_hm_1(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]) { register_hm_row<1>(tab); }
} // namespace gci
