// eri_kf_d.cu -- ket-first ERI class kernels with bra pair type [9].
#include "eri_classes.cuh"

namespace gci {
void register_eri_kf_d(LaunchFn (*tab)[kNumPairTypes][kNumPairTypes])
{
    register_row_kf_all<9>(tab);
}
} // namespace gci
