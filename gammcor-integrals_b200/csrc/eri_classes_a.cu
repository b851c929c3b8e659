// eri_classes_a.cu -- team ERI class kernels with bra pair types [0, 1, 2, 3, 4, 5]
// (s, p and d bras).  Classes with an f shell in the bra use the ket-first
// kernels only: the team kernel never won the per-class timing there.
#include "eri_classes.cuh"

namespace gci {
void register_eri_classes_a(LaunchFn (*tab)[kNumPairTypes])
{
    register_row<0>(tab);
    register_row<1>(tab);
    register_row<2>(tab);
    register_row<3>(tab);
    register_row<4>(tab);
    register_row<5>(tab);
}
} // namespace gci
