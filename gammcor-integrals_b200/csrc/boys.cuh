// boys.cuh -- device Boys function F_0..F_m(x) in FP64.
//
// Same scheme as the reference (src/integrals/boys.f90:202-281): x < 25 ->
// 5-point Chebyshev interpolation of F_m on one of 500 intervals
// (cheb_approx_5, chebinterp.f90:122-149), then downward recursion
// F_{k-1} = (2x F_k + e^{-x}) / (2k-1); x >= 25 -> F_0 = sqrt(pi/x)/2 and
// upward recursion.  The coefficient table is built on the host
// (boys_table.cpp) and read through the read-only data path.
#pragma once
#include "gci_common.h"

namespace gci {

template <int M>
__device__ __forceinline__ void boys_fm(double x, const double* __restrict__ table, double (&F)[M + 1])
{
    if (x < kBoysXAsym) {
        const int k = static_cast<int>(x * (1.0 / kBoysDelta));
        const int kk = k < kBoysNInt ? k : kBoysNInt - 1;
        const double* c = table + (static_cast<size_t>(M) * kBoysNInt + kk) * 5;
        const double ab_sum = static_cast<double>(2 * kk + 1) * kBoysDelta;
        const double y = (2.0 * x - ab_sum) * (1.0 / kBoysDelta);
        const double twoy = 2.0 * y;
        const double d5 = __ldg(c + 4);
        const double d4 = twoy * d5 + __ldg(c + 3);
        const double d3 = twoy * d4 - d5 + __ldg(c + 2);
        const double d2 = twoy * d3 - d4 + __ldg(c + 1);
        double f = y * d2 - d3 + 0.5 * __ldg(c + 0);
        F[M] = f;
        if constexpr (M > 0) {
            const double expmx = exp(-x);
            const double twox = 2.0 * x;
#pragma unroll
            for (int l = M; l >= 1; --l) {
                f = (twox * f + expmx) * (1.0 / static_cast<double>(2 * l - 1));
                F[l - 1] = f;
            }
        }
    } else {
        double f = 0.5 * sqrt(kPi / x);
        F[0] = f;
        if constexpr (M > 0) {
            const double expmx = exp(-x);
            const double beta = 1.0 / (2.0 * x);
#pragma unroll
            for (int l = 1; l <= M; ++l) {
                f = beta * (static_cast<double>(2 * l - 1) * f - expmx);
                F[l] = f;
            }
        }
    }
}

// Runtime-order variant used by the Boys self-test entry point.
__device__ __forceinline__ void boys_fm_rt(int m, double x, const double* __restrict__ table, double* F)
{
    if (x < kBoysXAsym) {
        const int k = static_cast<int>(x * (1.0 / kBoysDelta));
        const int kk = k < kBoysNInt ? k : kBoysNInt - 1;
        const double* c = table + (static_cast<size_t>(m) * kBoysNInt + kk) * 5;
        const double ab_sum = static_cast<double>(2 * kk + 1) * kBoysDelta;
        const double y = (2.0 * x - ab_sum) * (1.0 / kBoysDelta);
        const double twoy = 2.0 * y;
        const double d5 = c[4];
        const double d4 = twoy * d5 + c[3];
        const double d3 = twoy * d4 - d5 + c[2];
        const double d2 = twoy * d3 - d4 + c[1];
        double f = y * d2 - d3 + 0.5 * c[0];
        F[m] = f;
        const double expmx = exp(-x), twox = 2.0 * x;
        for (int l = m; l >= 1; --l) {
            f = (twox * f + expmx) / static_cast<double>(2 * l - 1);
            F[l - 1] = f;
        }
    } else {
        double f = 0.5 * sqrt(kPi / x);
        F[0] = f;
        const double expmx = exp(-x), beta = 1.0 / (2.0 * x);
        for (int l = 1; l <= m; ++l) {
            f = beta * (static_cast<double>(2 * l - 1) * f - expmx);
            F[l] = f;
        }
    }
}

} // namespace gci
