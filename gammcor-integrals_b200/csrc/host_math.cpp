// host_math.cpp -- host-side numerics of the library: the Boys interpolation
// table, real-solid-harmonic coefficients, basis normalisation and the SLATEC
// sort used by the pivot bookkeeping.
#include "host_math.h"
#include <cmath>
#include <cstring>
#include <vector>

namespace gci {

// Shavitt series for F_m (boys.f90:166-199), denominator in floating point.
static double shavitt(int m, double twox, double expmx)
{
    double sum = 0.0, xi = 1.0, a = 2.0 * m + 1.0, d = a;
    for (int i = 0; i < 6; ++i) {
        sum += xi / d;
        xi *= twox;
        a += 2.0;
        d *= a;
    }
    return expmx * sum;
}

// High-accuracy F_m(x) used to sample the interpolation nodes (fm_reference,
// boys.f90:94-163): series far above m, then the stable downward recursion.
double boys_reference(int m, double x)
{
    if (x < 35.0) {
        int dm = x < 1.0 ? 15 : x < 5.0 ? 30 : x < 10.0 ? 50 : x < 15.0 ? 60 : x < 20.0 ? 70 : x < 25.0 ? 80
               : x < 30.0 ? 90 : 100;
        const double expmx = std::exp(-x), twox = 2.0 * x;
        double f = shavitt(m + dm, twox, expmx);
        int a = 2 * (m + dm - 1) + 1;
        for (int l = 1; l <= dm; ++l) {
            f = 1.0 / (double)a * (twox * f + expmx);
            a -= 2;
        }
        return f;
    }
    double f = 0.5 * std::sqrt(kPi / x);
    const double expmx = std::exp(-x), beta = 1.0 / (2.0 * x);
    int a = 1;
    for (int l = 2; l <= m + 1; ++l) {
        f = beta * ((double)a * f - expmx);
        a += 2;
    }
    return f;
}

// 5-point Chebyshev coefficients of F_m on 500 intervals of [0, 25)
// (boys_init boys.f90:57-86; cheb_nodes/cheb_coeffs chebinterp.f90:9-56).
std::vector<double> boys_table(int maxm)
{
    const int n = 5;
    std::vector<double> tab((size_t)(maxm + 1) * kBoysNInt * n);
    const double w0 = kPi / n;
    for (int k = 0; k <= maxm; ++k)
        for (int i = 0; i < kBoysNInt; ++i) {
            const double a = i * kBoysDelta, b = (i + 1) * kBoysDelta;
            const double w1 = (b - a) / 2.0, w2 = (b + a) / 2.0;
            double fs[5];
            for (int j = 0; j < n; ++j) fs[j] = boys_reference(k, w1 * std::cos(w0 * (j + 0.5)) + w2);
            double* c = tab.data() + ((size_t)k * kBoysNInt + i) * n;
            for (int j = 0; j < n; ++j) {
                double s = 0.0;
                for (int q = 0; q < n; ++q) s += fs[q] * std::cos(w0 * j * (q + 0.5));
                c[j] = 2.0 / n * s;
            }
        }
    return tab;
}

static double factorial(int n) { double r = 1.0; for (int i = 2; i <= n; ++i) r *= i; return r; }
static double choose(int n, int k)
{
    if (k < 0 || k > n) return 0.0;
    return factorial(n) / (factorial(k) * factorial(n - k));
}
static double dfact(int n) { double r = 1.0; for (int i = n; i > 1; i -= 2) r *= i; return r; }

// Real solid harmonics S_lm = N_lm sum_{t,u,v} C^{lm}_{tuv} x^{2t+|m|-2(u+v)} y^{2(u+v)} z^{l-2t-|m|}
// (Helgaker, Jorgensen, Olsen, Eqs. 6.4.47-6.4.50), normalised to one on the unit
// sphere -- the convention of the reference generator (AutoSpherTransf.py:59-140).
// Rows m = -L..L; columns in the Auto2e Cartesian order; identity for L < 2
// (SPHER_TRANSF_LMIN, Auto2eGlobal.py:26).
void spher_coeffs(int L, double* U)
{
    const int nc = ncart(L), ns = 2 * L + 1;
    std::memset(U, 0, sizeof(double) * nc * ns);
    if (L < 2) {
        for (int i = 0; i < nc; ++i) U[i * nc + i] = 1.0;
        return;
    }
    for (int m = -L; m <= L; ++m) {
        const int am = m < 0 ? -m : m;
        const int vm2 = m >= 0 ? 0 : 1;
        double nlm = std::sqrt(2.0 * factorial(L + am) * factorial(L - am) / (m == 0 ? 2.0 : 1.0)) /
                     (std::pow(2.0, am) * factorial(L));
        nlm *= std::sqrt((2.0 * L + 1.0) / (4.0 * kPi));
        for (int t = 0; t <= (L - am) / 2; ++t)
            for (int u = 0; u <= t; ++u)
                for (int k = 0; k <= (am - vm2) / 2; ++k) {
                    const int twov = 2 * k + vm2;
                    const double c = (((t + k) & 1) ? -1.0 : 1.0) * std::pow(0.25, t) * choose(L, t) *
                                     choose(L - t, am + t) * choose(t, u) * choose(am, twov);
                    const int ey = 2 * u + twov, ez = L - 2 * t - am;
                    U[(m + L) * nc + cart_pos(ey, ez)] += nlm * c;
                }
    }
}

// basis_NormalizeCntrCoeffs (basis_sets.f90:894-945) and
// SpherGTO_NormFactors_Shell / ShellOverlap (sphergto.f90:184-269).
void normalize_basis(int64_t nparams, int64_t ldprim, const int64_t* L, const int64_t* nprim, const double* exps,
                     double* coefs, double* norm_cart, int64_t ldcart, double* norm_spher, int64_t ldsph)
{
    for (int64_t a = 0; a < nparams; ++a) {
        const int l = (int)L[a];
        const int np = (int)nprim[a];
        const double* e = exps + a * ldprim;
        double* c = coefs + a * ldprim;
        for (int i = 0; i < np; ++i)
            c[i] *= std::pow(2.0 / kPi, 0.75) * std::pow(2.0, l) * std::pow(e[i], (2.0 * l + 3.0) / 4.0);
        double z = 0.0;
        for (int i = 0; i < np; ++i)
            for (int j = 0; j < np; ++j) z += c[i] * c[j] / std::pow(e[i] + e[j], l + 1.5);
        const double y = std::sqrt(std::pow(kPi, 1.5) / std::pow(2.0, l));
        z = std::sqrt(z);
        if (norm_cart) {
            for (int64_t v = 0; v < ldcart; ++v) norm_cart[a * ldcart + v] = 0.0;
            int v = 0;
            for (int lx = l; lx >= 0; --lx)
                for (int ly = l - lx; ly >= 0; --ly) {
                    const int lz = l - lx - ly;
                    const double x = std::sqrt(dfact(2 * lx - 1) * dfact(2 * ly - 1) * dfact(2 * lz - 1));
                    norm_cart[a * ldcart + v++] = 1.0 / (x * y * z);
                }
        }
        if (norm_spher) {
            const int nc = ncart(l), ns = 2 * l + 1;
            std::vector<double> S((size_t)nc * nc, 0.0), U((size_t)nc * ns);
            std::vector<int> cx(nc), cy(nc), cz(nc);
            int q = 0;
            for (int lx = l; lx >= 0; --lx)
                for (int ly = l - lx; ly >= 0; --ly) { cx[q] = lx; cy[q] = ly; cz[q] = l - lx - ly; ++q; }
            for (int p1 = 0; p1 < np; ++p1)
                for (int p2 = 0; p2 < np; ++p2) {
                    const double ap = e[p2] + e[p1];
                    double od[2 * 6 + 1] = {0};
                    for (int t = 0; t <= l; ++t) od[2 * t] = dfact(2 * t - 1) / std::pow(2.0 * ap, t) * std::sqrt(kPi / ap);
                    for (int j = 0; j < nc; ++j)
                        for (int i = 0; i < nc; ++i)
                            S[i + nc * j] += c[p2] * c[p1] * od[cx[i] + cx[j]] * od[cy[i] + cy[j]] * od[cz[i] + cz[j]];
                }
            spher_coeffs(l, U.data());
            for (int64_t v = 0; v < ldsph; ++v) norm_spher[a * ldsph + v] = 0.0;
            for (int m = 0; m < ns; ++m) {
                double s = 0.0;
                for (int i = 0; i < nc; ++i)
                    for (int j = 0; j < nc; ++j) s += U[m * nc + i] * S[i + nc * j] * U[m * nc + j];
                norm_spher[a * ldsph + m] = 1.0 / std::sqrt(s);
            }
        }
    }
}

// SLATEC DSORT (Singleton's quicksort with insertion sort for short
// segments), carrying an index array; kflag = 2 ascending, -2 descending.
// The reference sorts with this routine (sort.f90:19) and ties keep the
// order it produces, so the same steps are followed here.
void slatec_dsort(double* dx, int64_t* dy, int64_t n, int kflag)
{
    if (n <= 1) return;
    if (kflag <= -1)
        for (int64_t i = 0; i < n; ++i) dx[i] = -dx[i];
    double* X = dx - 1;
    int64_t* Y = dy - 1;
    int64_t il[64], iu[64];
    int64_t m = 1, i = 1, j = n, k, l, ij;
    double r = 0.375, t, tt;
    int64_t ty, tty;
    goto s110;
s110:
    if (i == j) goto s150;
    if (r <= 0.5898437) r += 3.90625e-2; else r -= 0.21875;
s120:
    k = i;
    ij = i + (int64_t)((double)(j - i) * r);
    t = X[ij]; ty = Y[ij];
    if (X[i] > t) { X[ij] = X[i]; X[i] = t; t = X[ij]; Y[ij] = Y[i]; Y[i] = ty; ty = Y[ij]; }
    l = j;
    if (X[j] < t) {
        X[ij] = X[j]; X[j] = t; t = X[ij]; Y[ij] = Y[j]; Y[j] = ty; ty = Y[ij];
        if (X[i] > t) { X[ij] = X[i]; X[i] = t; t = X[ij]; Y[ij] = Y[i]; Y[i] = ty; ty = Y[ij]; }
    }
s130:
    --l;
    if (X[l] > t) goto s130;
s140:
    ++k;
    if (X[k] < t) goto s140;
    if (k <= l) {
        tt = X[l]; X[l] = X[k]; X[k] = tt;
        tty = Y[l]; Y[l] = Y[k]; Y[k] = tty;
        goto s130;
    }
    if (l - i > j - k) { il[m - 1] = i; iu[m - 1] = l; i = k; ++m; }
    else { il[m - 1] = k; iu[m - 1] = j; j = l; ++m; }
    goto s160;
s150:
    --m;
    if (m == 0) goto s190;
    i = il[m - 1]; j = iu[m - 1];
s160:
    if (j - i >= 1) goto s120;
    if (i == 1) goto s110;
    --i;
s170:
    ++i;
    if (i == j) goto s150;
    t = X[i + 1]; ty = Y[i + 1];
    if (X[i] <= t) goto s170;
    k = i;
s180:
    X[k + 1] = X[k]; Y[k + 1] = Y[k];
    --k;
    if (t < X[k]) goto s180;
    X[k + 1] = t; Y[k + 1] = ty;
    goto s170;
s190:
    if (kflag <= -1)
        for (int64_t q = 0; q < n; ++q) dx[q] = -dx[q];
}

} // namespace gci
