// eri_hm_4.cu -- Hermite-matrix ERI kernels with row pairs of Hermite level 4.
#include "eri_hermite.cuh"

namespace gci {
void register_hm_4(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]) { register_hm_row<4>(tab); }
} // namespace gci
