// grad_pot_c.cu -- Coulomb-potential kernels of the adjoint path for the
// level classes with L1 + L2 in 10..12 (grad_engine.cuh).
#include "grad_engine.cuh"
#include "gci_runtime.h"

namespace gci {
void register_grad_pot_c(GradLaunchFn (*tab)[kGradMaxL + 1])
{
    register_grad_range<10, 12>(tab, std::make_integer_sequence<int, kGradMaxL + 1>{});
}
} // namespace gci
