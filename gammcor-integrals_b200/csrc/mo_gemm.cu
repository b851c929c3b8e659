// mo_gemm.cu -- split-precision tensor-core GEMMs (see mo_gemm.h).
#include "mo_gemm.h"

namespace gci {
cudaError_t mo_gemm_mixed(const double*, int64_t, int64_t, int64_t, const double*, double*, cudaStream_t)
{
    return cudaErrorNotSupported;
}
cudaError_t mo_gemm_mixed_batched(const double*, int64_t, int64_t, int64_t, const double*, double*, int64_t, int64_t,
                                  cudaStream_t)
{
    return cudaErrorNotSupported;
}
} // namespace gci
