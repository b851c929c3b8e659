// eri_kf_a.cu -- ket-first ERI class kernels with bra pair types [3, 4, 5].
#include "eri_classes.cuh"

namespace gci {
void register_eri_kf_a(LaunchFn (*tab)[kNumPairTypes][kNumPairTypes])
{
    register_row_kf_all<3>(tab);
    register_row_kf_all<4>(tab);
    register_row_kf_all<5>(tab);
}
} // namespace gci
