// eri_classes_b.cu -- ERI class kernels with bra pair types [6, 7].
#include "eri_classes.cuh"

namespace gci {
void register_eri_classes_b(LaunchFn (*tab)[kNumPairTypes])
{
    register_row<6>(tab);
    register_row<7>(tab);
}
} // namespace gci
