// eri_classes_c.cu -- ERI class kernels with bra pair types [8].
#include "eri_classes.cuh"

namespace gci {
void register_eri_classes_c(LaunchFn (*tab)[kNumPairTypes])
{
    register_row<8>(tab);
}
} // namespace gci
