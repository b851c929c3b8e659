// eri_hm_2.cu -- Hermite-matrix ERI kernels with row pairs of Hermite level 2.
#include "eri_hermite.cuh"

namespace gci {
void register_hm_2(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]) { register_hm_row<2>(tab); }
} // namespace gci
