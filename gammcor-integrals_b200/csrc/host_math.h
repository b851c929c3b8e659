// host_math.h -- host numerics shared by the runtime (see host_math.cpp).
#pragma once
#include "gci_common.h"
#include <vector>

namespace gci {
double boys_reference(int m, double x);
std::vector<double> boys_table(int maxm);
void spher_coeffs(int L, double* U);
void normalize_basis(int64_t nparams, int64_t ldprim, const int64_t* L, const int64_t* nprim, const double* exps,
                     double* coefs, double* norm_cart, int64_t ldcart, double* norm_spher, int64_t ldsph);
void slatec_dsort(double* dx, int64_t* dy, int64_t n, int kflag);
} // namespace gci
