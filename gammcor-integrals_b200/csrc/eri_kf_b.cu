// eri_kf_b.cu -- ket-first ERI class kernels with bra pair types [6, 7].
#include "eri_classes.cuh"

namespace gci {
void register_eri_kf_b(LaunchFn (*tab)[kNumPairTypes][kNumPairTypes])
{
    register_row_kf_all<6>(tab);
    register_row_kf_all<7>(tab);
}
} // namespace gci
