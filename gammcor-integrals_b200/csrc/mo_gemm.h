// mo_gemm.h -- split-precision tensor-core GEMMs for the AO->MO transformation.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace gci {
// C(m x n) = A(m x k) B(k x n), all FP64 column-major with lda = m, ldb = k, ldc = m.
cudaError_t mo_gemm_mixed(const double* A, int64_t m, int64_t n, int64_t k, const double* B, double* C,
                          cudaStream_t s);
// for a in [0, batch): C + a*ldc_batch (kc x n, ld = ldk*batch) = A_a(kc x k, ld kc, stride kc*k) B(k x n)
cudaError_t mo_gemm_mixed_batched(const double* A, int64_t kc, int64_t n, int64_t k, const double* B, double* C,
                                  int64_t ldk, int64_t batch, cudaStream_t s);
} // namespace gci
