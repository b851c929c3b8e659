// eri_classes_d.cu -- ERI class kernels with bra pair types [9].
#include "eri_classes.cuh"

namespace gci {
void register_eri_classes_d(LaunchFn (*tab)[kNumPairTypes])
{
    register_row<9>(tab);
}
} // namespace gci
