// eri_hm_6.cu -- Hermite-matrix ERI kernels with row pairs of Hermite level 6.
#include "eri_hermite.cuh"

namespace gci {
void register_hm_6(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]) { register_hm_row<6>(tab); }
} // namespace gci
