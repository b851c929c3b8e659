// eri_kf_c.cu -- ket-first ERI class kernels with bra pair type [8].
#include "eri_classes.cuh"

namespace gci {
void register_eri_kf_c(LaunchFn (*tab)[kNumPairTypes][kNumPairTypes])
{
    register_row_kf_all<8>(tab);
}
} // namespace gci
