/*
 * gci_oracle.c -- FP64 CPU oracle for the integral-direct two-step Cholesky
 * decomposition of (pq|rs) and the AO->MO transformation of the vectors.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU legs may load it.
 *
 * Every routine restates the reference algorithm (modrzejewski/
 * gammcor-integrals); the file:line it follows is given at each function.
 * Parity pins and their limits are listed in gci_oracle.h.
 */
#include "gci_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI 3.14159265358979323846264338327950288
#define MAXLEV (2 * ORC_MAXL + 1)          /* highest bra/ket level incl. derivative shift */
#define MAXLT (2 * MAXLEV)                 /* highest total Hermite level  */
#define CART_OFF(l) ((l) * ((l) + 1) * ((l) + 2) / 6)
#define NCART(l) (((l) + 1) * ((l) + 2) / 2)
#define HERM_N(n) (((n) + 1) * ((n) + 2) * ((n) + 3) / 6)

static inline int herm_idx(int t, int u, int v)
{
    int n = t + u + v, s = u + v;
    return n * (n + 1) * (n + 2) / 6 + s * (s + 1) / 2 + v;
}
static inline int cart_pos(int ly, int lz) { int s = ly + lz; return s * (s + 1) / 2 + lz; }

/* Cartesian components, global index CART_OFF(l) + position, in the Auto2e
 * order: lx descending, then ly descending (Auto2eGlobal.py:35-44,
 * basis_sets.f90:797-806). */
static int g_cx[CART_OFF(MAXLEV + 2)], g_cy[CART_OFF(MAXLEV + 2)], g_cz[CART_OFF(MAXLEV + 2)];

__attribute__((constructor)) static void orc_tables_init(void)
{
    for (int l = 0; l <= MAXLEV + 1; ++l) {
        int i = CART_OFF(l);
        for (int x = l; x >= 0; --x)
            for (int y = l - x; y >= 0; --y) {
                g_cx[i] = x; g_cy[i] = y; g_cz[i] = l - x - y; ++i;
            }
    }
}

/* ====================================================================== */
/* Boys function                                                          */
/* ====================================================================== */
#define BOYS_NINT 500              /* NINTERVALS_CHEB5(3), boys.f90:20-21,43 */
#define BOYS_XASYM 25.0            /* X_ASYMPTOTIC_CHEB5(3)                  */
#define BOYS_DELTAX (BOYS_XASYM / BOYS_NINT)
static double *g_boys = NULL;      /* [m][interval][5] */
static int g_boys_maxm = -1;

/* Shavitt series, boys.f90:166-199.  The reference evaluates the running
 * denominator in default (32-bit) integers, which overflows for orders above
 * ~15; here it is evaluated in floating point (the difference is damped by
 * the downward recursion to below 1e-15 relative). */
static double fm_shavitt(int m, double twox, double expmx)
{
    double sum = 0.0, xi = 1.0, d = 2.0 * m + 1.0, a = 2.0 * m + 1.0;
    for (int i = 0; i < 6; ++i) {
        sum += xi / d;
        xi *= twox;
        a += 2.0;
        d *= a;
    }
    return expmx * sum;
}

/* fm_reference, boys.f90:94-163 */
double orc_fm_reference(int m, double x)
{
    double f;
    if (x < 35.0) {
        int dm;
        if (x < 1.0) dm = 15; else if (x < 5.0) dm = 30; else if (x < 10.0) dm = 50;
        else if (x < 15.0) dm = 60; else if (x < 20.0) dm = 70; else if (x < 25.0) dm = 80;
        else if (x < 30.0) dm = 90; else dm = 100;
        double expmx = exp(-x), twox = 2.0 * x;
        f = fm_shavitt(m + dm, twox, expmx);
        int a = 2 * (m + dm - 1) + 1;
        for (int l = 1; l <= dm; ++l) {
            f = 1.0 / (double)a * (twox * f + expmx);
            a -= 2;
        }
    } else {
        f = 0.5 * sqrt(PI / x);
        double expmx = exp(-x), beta = 1.0 / (2.0 * x);
        int a = 1;
        for (int l = 2; l <= m + 1; ++l) {
            f = beta * ((double)a * f - expmx);
            a += 2;
        }
    }
    return f;
}

/* cheb_nodes / cheb_coeffs, chebinterp.f90:9-56; boys_init boys.f90:57-86 */
int orc_boys_init(int maxm)
{
    if (maxm < 0 || maxm > 4 * MAXLEV) return -1;
    if (g_boys && g_boys_maxm >= maxm) return 0;
    double *tab = (double *)malloc(sizeof(double) * (size_t)(maxm + 1) * BOYS_NINT * 5);
    if (!tab) return -2;
    const int n = 5;
    for (int k = 0; k <= maxm; ++k)
        for (int i = 0; i < BOYS_NINT; ++i) {
            double a = i * BOYS_DELTAX, b = (i + 1) * BOYS_DELTAX;
            double xs[5], fs[5];
            double w0 = PI / n, w1 = (b - a) / 2.0, w2 = (b + a) / 2.0;
            for (int j = 0; j < n; ++j) {
                xs[j] = w1 * cos(w0 * (j + 1 - 0.5)) + w2;
                fs[j] = orc_fm_reference(k, xs[j]);
            }
            double *c = tab + ((size_t)k * BOYS_NINT + i) * 5;
            for (int j = 0; j < n; ++j) {
                double s = 0.0;
                for (int q = 0; q < n; ++q) s += fs[q] * cos(w0 * j * (q + 1 - 0.5));
                c[j] = 2.0 / n * s;
            }
        }
    free(g_boys);
    g_boys = tab;
    g_boys_maxm = maxm;
    return 0;
}

/* fm_interp boys.f90:202-221 + cheb_approx_5 chebinterp.f90:122-149 */
static double fm_interp(double x, int m)
{
    int k = (int)floor(x / BOYS_DELTAX);
    double ab_sum = (double)(2 * k + 1) * BOYS_DELTAX;
    const double *c = g_boys + ((size_t)m * BOYS_NINT + k) * 5;
    double y = (2.0 * x - ab_sum) / BOYS_DELTAX, twoy = 2.0 * y;
    double d5 = c[4];
    double d4 = twoy * d5 + c[3];
    double d3 = twoy * d4 - d5 + c[2];
    double d2 = twoy * d3 - d4 + c[1];
    return y * d2 - d3 + 0.5 * c[0];
}

/* fm, boys.f90:224-281: F_0..F_m */
void orc_fm(int m, double x, double *fm)
{
    if (x < BOYS_XASYM) {
        double f = fm_interp(x, m);
        fm[m] = f;
        double expmx = exp(-x), twox = 2.0 * x, a = (double)(2 * (m - 1) + 1);
        for (int l = m; l >= 1; --l) {
            f = (twox * f + expmx) / a;
            fm[l - 1] = f;
            a -= 2.0;
        }
    } else {
        double f = 0.5 * sqrt(PI / x);
        fm[0] = f;
        double expmx = exp(-x), a = 1.0, beta = 1.0 / (2.0 * x);
        for (int l = 2; l <= m + 1; ++l) {
            f = beta * (a * f - expmx);
            a += 2.0;
            fm[l - 1] = f;
        }
    }
}

void orc_fm_batch(int m, int64_t n, const double *x, double *out)
{
    for (int64_t i = 0; i < n; ++i) orc_fm(m, x[i], out + i * (m + 1));
}

/* ====================================================================== */
/* Real solid harmonics and normalisation                                 */
/* ====================================================================== */
static double fact(int n) { double r = 1.0; for (int i = 2; i <= n; ++i) r *= i; return r; }
static double binom(int n, int k)
{
    if (k < 0 || k > n) return 0.0;
    return fact(n) / (fact(k) * fact(n - k));
}
static double dblfact(int n) { double r = 1.0; for (int i = n; i > 1; i -= 2) r *= i; return r; }

/* Cartesian -> real spherical harmonic coefficients for one shell: the
 * published real solid harmonic expansion (Helgaker, Jorgensen, Olsen,
 * Eqs. 6.4.47-6.4.50) scaled to unit norm on the sphere, as generated by the
 * reference in AutoSpherTransf.py:59-160.  Rows m = -L..L, columns the
 * Cartesian order above.  L < 2 stays Cartesian (Auto2eGlobal.py:26). */
void orc_spher_u(int L, double *U)
{
    int nc = NCART(L), ns = 2 * L + 1;
    memset(U, 0, sizeof(double) * nc * ns);
    if (L < 2) {
        for (int i = 0; i < nc; ++i) U[i * nc + i] = 1.0;
        return;
    }
    for (int m = -L; m <= L; ++m) {
        int am = abs(m);
        int vm2 = (m >= 0) ? 0 : 1;        /* 2 v_m */
        double nlm = sqrt(2.0 * fact(L + am) * fact(L - am) / (m == 0 ? 2.0 : 1.0)) /
                     (pow(2.0, am) * fact(L));
        nlm *= sqrt((2.0 * L + 1.0) / (4.0 * PI));
        for (int t = 0; t <= (L - am) / 2; ++t)
            for (int u = 0; u <= t; ++u)
                for (int k = 0; k <= (am - vm2) / 2; ++k) {
                    int twov = 2 * k + vm2;   /* 2v, v = v_m + k */
                    double c = (((t + k) & 1) ? -1.0 : 1.0) * pow(0.25, t) * binom(L, t) *
                               binom(L - t, am + t) * binom(t, u) * binom(am, twov);
                    /* x^{2t+|m|-2(u+v)} y^{2(u+v)} z^{l-2t-|m|} */
                    int ey = 2 * u + twov, ez = L - 2 * t - am;
                    U[(m + L) * nc + cart_pos(ey, ez)] += nlm * c;
                }
    }
}

/* basis_NormalizeCntrCoeffs, basis_sets.f90:894-945 */
void orc_normalize_cntr(int nparams, int ldprim, const int *L, const int *nprim,
                        const double *exps, double *coefs, double *normcart, int ldcart)
{
    for (int a = 0; a < nparams; ++a) {
        int np = nprim[a], l = L[a];
        const double *e = exps + (size_t)a * ldprim;
        double *c = coefs + (size_t)a * ldprim;
        for (int i = 0; i < np; ++i)
            c[i] *= pow(2.0 / PI, 0.75) * pow(2.0, l) * pow(e[i], (2.0 * l + 3.0) / 4.0);
        double z = 0.0;
        for (int i = 0; i < np; ++i)
            for (int j = 0; j < np; ++j)
                z += c[i] * c[j] / pow(e[i] + e[j], l + 1.5);
        double y = sqrt(pow(PI, 1.5) / pow(2.0, l));
        z = sqrt(z);
        for (int v = 0; v < ldcart; ++v) normcart[(size_t)a * ldcart + v] = 0.0;
        int v = 0;
        for (int lx = l; lx >= 0; --lx)
            for (int ly = l - lx; ly >= 0; --ly) {
                int lz = l - lx - ly;
                double x = sqrt(dblfact(2 * lx - 1) * dblfact(2 * ly - 1) * dblfact(2 * lz - 1));
                normcart[(size_t)a * ldcart + v] = 1.0 / (x * y * z);
                ++v;
            }
    }
}

/* SpherGTO_NormFactors_Shell + ShellOverlap, sphergto.f90:166-269 */
void orc_spher_norms(int nparams, int ldprim, const int *L, const int *nprim,
                     const double *exps, const double *coefs, double *normspher, int ldsph)
{
    for (int a = 0; a < nparams; ++a) {
        int l = L[a], np = nprim[a], nc = NCART(l), ns = 2 * l + 1;
        const double *e = exps + (size_t)a * ldprim;
        const double *c = coefs + (size_t)a * ldprim;
        double *S = (double *)calloc((size_t)nc * nc, sizeof(double));
        double *U = (double *)malloc(sizeof(double) * nc * ns);
        int base = CART_OFF(l);
        for (int q = 0; q < np; ++q)
            for (int k = 0; k < np; ++k) {
                double ap = e[k] + e[q];
                double od[2 * ORC_MAXL + 1];
                for (int t = 0; t <= 2 * l; ++t) od[t] = 0.0;
                for (int t = 0; t <= l; ++t)
                    od[2 * t] = dblfact(2 * t - 1) / pow(2.0 * ap, t) * sqrt(PI / ap);
                for (int j = 0; j < nc; ++j)
                    for (int i = 0; i < nc; ++i)
                        S[i + nc * j] += c[k] * c[q] * od[g_cx[base + i] + g_cx[base + j]] *
                                         od[g_cy[base + i] + g_cy[base + j]] *
                                         od[g_cz[base + i] + g_cz[base + j]];
            }
        orc_spher_u(l, U);
        for (int v = 0; v < ldsph; ++v) normspher[(size_t)a * ldsph + v] = 0.0;
        for (int m = 0; m < ns; ++m) {
            double s = 0.0;
            for (int i = 0; i < nc; ++i)
                for (int j = 0; j < nc; ++j) s += U[m * nc + i] * S[i + nc * j] * U[m * nc + j];
            normspher[(size_t)a * ldsph + m] = 1.0 / sqrt(s);
        }
        free(S); free(U);
    }
}

/* ====================================================================== */
/* Shell-quartet ERI: W-matrix (LS|KS) + HRR + transform                   */
/* ====================================================================== */

/* Single-centre Hermite coefficients E^{e}_t, e <= emax, for the Gaussian
 * (x-A)^e exp(-p (x-P)^2): the McMurchie-Davidson recursion with the
 * second index zero (auto2e_EtCoeffs_L, auto2e_Hermite.f90:10-423). */
static void et_coeffs(int emax, double p, double X, double *E /* [emax+1][emax+1] */)
{
    int ld = emax + 1;
    for (int i = 0; i < ld * ld; ++i) E[i] = 0.0;
    E[0] = 1.0;
    double h = 1.0 / (2.0 * p);
    for (int e = 0; e < emax; ++e)
        for (int t = 0; t <= e + 1; ++t) {
            double v = 0.0;
            if (t >= 1) v += h * E[e * ld + t - 1];
            if (t <= e) v += X * E[e * ld + t];
            if (t + 1 <= e) v += (t + 1) * E[e * ld + t + 1];
            E[(e + 1) * ld + t] = v;
        }
}

/* Hermite Coulomb integrals R_tuv, t+u+v <= n (auto2e_Rtuv_n,
 * auto2e_Hermite.f90:11330-11878; recursion rules Auto2e.py:80-119). */
static void rtuv(int n, const double *F, double alpha, double X, double Y, double Z, double *R)
{
    static __thread double buf[2][HERM_N(MAXLT)];
    double *cur = buf[0], *nxt = buf[1];
    double m2a = -2.0 * alpha;
    /* level j = n: only R^{(n)}_000 */
    double pw = 1.0;
    double pows[MAXLT + 1];
    for (int j = 0; j <= n; ++j) { pows[j] = pw; pw *= m2a; }
    cur[0] = pows[n] * F[n];
    for (int j = n - 1; j >= 0; --j) {
        int top = n - j;
        for (int k = 0; k <= top; ++k)
            for (int s = 0; s <= k; ++s)
                for (int v = 0; v <= s; ++v) {
                    int u = s - v, t = k - s;
                    double r;
                    if (t >= 1) {
                        r = X * cur[herm_idx(t - 1, u, v)];
                        if (t >= 2) r += (t - 1) * cur[herm_idx(t - 2, u, v)];
                    } else if (u >= 1) {
                        r = Y * cur[herm_idx(t, u - 1, v)];
                        if (u >= 2) r += (u - 1) * cur[herm_idx(t, u - 2, v)];
                    } else if (v >= 1) {
                        r = Z * cur[herm_idx(t, u, v - 1)];
                        if (v >= 2) r += (v - 1) * cur[herm_idx(t, u, v - 2)];
                    } else {
                        r = pows[j] * F[j];
                    }
                    nxt[herm_idx(t, u, v)] = r;
                }
        double *tmp = cur; cur = nxt; nxt = tmp;
    }
    memcpy(R, cur, sizeof(double) * HERM_N(n));
}

/* W(e,f) = (e0|f0) summed over primitives, e in levels la..la+lb on centre
 * A, f in levels lc..lc+ld on centre C.  Loop order and prefactors follow
 * auto2e_W_L_K, e.g. auto2e_WMatrix_part1.f90:743-812 (Kappa: erf-attenuated
 * operator, Alpha = PQ/(P+Q+Kappa PQ)). */
static void wmatrix(int la, int lb, int lc, int ld,
                    const double *Ra, const double *Rb, const double *Rc, const double *Rd,
                    int na, const double *ea, const double *ca,
                    int nb, const double *eb, const double *cb,
                    int nc, const double *ec, const double *cc,
                    int nd, const double *ed, const double *cd,
                    double kappa, double *W /* [ne][nf] row-major */)
{
    int L1 = la + lb, L2 = lc + ld, LT = L1 + L2;
    int e0 = CART_OFF(la), e1 = CART_OFF(L1 + 1), f0 = CART_OFF(lc), f1 = CART_OFF(L2 + 1);
    int ne = e1 - e0, nf = f1 - f0;
    memset(W, 0, sizeof(double) * ne * nf);
    double Rab2 = 0, Rcd2 = 0;
    for (int i = 0; i < 3; ++i) {
        Rab2 += (Ra[i] - Rb[i]) * (Ra[i] - Rb[i]);
        Rcd2 += (Rc[i] - Rd[i]) * (Rc[i] - Rd[i]);
    }
    double Eab[3][(MAXLEV + 1) * (MAXLEV + 1)], Ecd[3][(MAXLEV + 1) * (MAXLEV + 1)];
    double F[MAXLT + 1];
    double *R = (double *)malloc(sizeof(double) * HERM_N(LT));
    double *S = (double *)malloc(sizeof(double) * HERM_N(L1));
    int l1p = L1 + 1, l2p = L2 + 1;
    for (int gd = 0; gd < nd; ++gd)
        for (int gc = 0; gc < nc; ++gc) {
            double Q = ec[gc] + ed[gd];
            double mucd = ec[gc] * ed[gd] / Q;
            double Rq[3], Rqc[3];
            for (int i = 0; i < 3; ++i) { Rq[i] = (ec[gc] * Rc[i] + ed[gd] * Rd[i]) / Q; Rqc[i] = Rq[i] - Rc[i]; }
            for (int i = 0; i < 3; ++i) et_coeffs(L2, Q, Rqc[i], Ecd[i]);
            for (int gb = 0; gb < nb; ++gb)
                for (int ga = 0; ga < na; ++ga) {
                    double P = ea[ga] + eb[gb];
                    double muab = ea[ga] * eb[gb] / P;
                    double Rp[3], Rpa[3], Rpq[3];
                    for (int i = 0; i < 3; ++i) {
                        Rp[i] = (ea[ga] * Ra[i] + eb[gb] * Rb[i]) / P;
                        Rpa[i] = Rp[i] - Ra[i];
                        Rpq[i] = Rp[i] - Rq[i];
                    }
                    double kabcd = exp(-muab * Rab2 - mucd * Rcd2);
                    double PQ = P * Q;
                    double alpha = PQ / (P + Q + kappa * PQ);
                    double N = 2.0 * pow(PI, 2.5) / (PQ * sqrt(P + Q + kappa * PQ));
                    double e000 = N * ca[ga] * cb[gb] * cc[gc] * cd[gd] * kabcd;
                    for (int i = 0; i < 3; ++i) et_coeffs(L1, P, Rpa[i], Eab[i]);
                    double T = alpha * (Rpq[0] * Rpq[0] + Rpq[1] * Rpq[1] + Rpq[2] * Rpq[2]);
                    orc_fm(LT, T, F);
                    rtuv(LT, F, alpha, Rpq[0], Rpq[1], Rpq[2], R);
                    for (int f = f0; f < f1; ++f) {
                        int fx = g_cx[f], fy = g_cy[f], fz = g_cz[f];
                        /* ket Hermite -> Cartesian with sign (-1)^{tau+nu+phi}
                         * (auto2e_KetTransform_*, e.g. _2_1.f90:20-25) */
                        for (int k = 0; k <= L1; ++k)
                            for (int s = 0; s <= k; ++s)
                                for (int v = 0; v <= s; ++v) {
                                    int u = s - v, t = k - s;
                                    double acc = 0.0;
                                    for (int p3 = 0; p3 <= fz; ++p3)
                                        for (int p2 = 0; p2 <= fy; ++p2)
                                            for (int p1 = 0; p1 <= fx; ++p1) {
                                                double sg = ((p1 + p2 + p3) & 1) ? -1.0 : 1.0;
                                                acc += sg * Ecd[0][fx * l2p + p1] * Ecd[1][fy * l2p + p2] *
                                                       Ecd[2][fz * l2p + p3] * R[herm_idx(t + p1, u + p2, v + p3)];
                                            }
                                    S[herm_idx(t, u, v)] = acc;
                                }
                        /* bra Hermite -> Cartesian (auto2e_BraTransform.f90) */
                        for (int e = e0; e < e1; ++e) {
                            int ex = g_cx[e], ey = g_cy[e], ez = g_cz[e];
                            double acc = 0.0;
                            for (int v = 0; v <= ez; ++v)
                                for (int u = 0; u <= ey; ++u)
                                    for (int t = 0; t <= ex; ++t)
                                        acc += Eab[0][ex * l1p + t] * Eab[1][ey * l1p + u] *
                                               Eab[2][ez * l1p + v] * S[herm_idx(t, u, v)];
                            W[(e - e0) * nf + (f - f0)] += e000 * acc;
                        }
                    }
                }
        }
    free(R); free(S);
}

/* Horizontal recurrence (Head-Gordon & Pople, Eq. 18) for one index pair:
 * in[f] for f in levels l1..l1+l2 (global Cartesian index minus CART_OFF(l1))
 * -> out[c + n1*d], c of level l1, d of level l2; AB = centre1 - centre2.
 * auto2e_KetTransfer.f90:12-34 applied as in auto2e_eri_dpdp.f90:98-117. */
static void hrr_pair(int l1, int l2, const double AB[3], const double *in, double *out)
{
    int n1 = NCART(l1);
    if (l2 == 0) { memcpy(out, in, sizeof(double) * n1); return; }
    int fo = CART_OFF(l1);
    int nfg = CART_OFF(l1 + l2 + 1);
    /* cur[(fglob) * nd + dpos] for d of current level k */
    double *cur = (double *)malloc(sizeof(double) * nfg * NCART(l2));
    double *nxt = (double *)malloc(sizeof(double) * nfg * NCART(l2));
    for (int f = fo; f < nfg; ++f) cur[f] = in[f - fo];
    for (int k = 0; k < l2; ++k) {
        int ndk = NCART(k), ndn = NCART(k + 1), dko = CART_OFF(k), dno = CART_OFF(k + 1);
        int ftop = CART_OFF(l1 + l2 - k);   /* f levels l1..l1+l2-k-1 */
        for (int f = fo; f < ftop; ++f)
            for (int dn = 0; dn < ndn; ++dn) {
                int dx = g_cx[dno + dn], dy = g_cy[dno + dn], dz = g_cz[dno + dn];
                int ax = (dx > 0) ? 0 : ((dy > 0) ? 1 : 2);
                int ddx = dx - (ax == 0), ddy = dy - (ax == 1), ddz = dz - (ax == 2);
                int dpos = cart_pos(ddy, ddz);
                int fx = g_cx[f] + (ax == 0), fy = g_cy[f] + (ax == 1), fz = g_cz[f] + (ax == 2);
                int fl = fx + fy + fz;
                int f1 = CART_OFF(fl) + cart_pos(fy, fz);
                (void)dko;
                nxt[f * ndn + dn] = cur[f1 * ndk + dpos] + AB[ax] * cur[f * ndk + dpos];
            }
        double *t = cur; cur = nxt; nxt = t;
    }
    int nd = NCART(l2);
    for (int c = 0; c < n1; ++c)
        for (int d = 0; d < nd; ++d) out[c + n1 * d] = cur[(fo + c) * nd + d];
    free(cur); free(nxt);
}

/* Contracted Cartesian (ab|cd), a fastest, from the W matrix: ket HRR, then
 * bra HRR (auto2e_BraKetTransfer_*, auto2e_eri_dpdp.f90:98-142). */
static void cart_quartet(int la, int lb, int lc, int ld,
                         const double *Ra, const double *Rb, const double *Rc, const double *Rd,
                         int na, const double *ea, const double *ca,
                         int nb, const double *eb, const double *cb,
                         int nc, const double *ec, const double *cc,
                         int nd, const double *ed, const double *cd,
                         double kappa, double *G)
{
    int ne = CART_OFF(la + lb + 1) - CART_OFF(la), nf = CART_OFF(lc + ld + 1) - CART_OFF(lc);
    int Na = NCART(la), Nb = NCART(lb), Nc = NCART(lc), Nd = NCART(ld);
    double *W = (double *)malloc(sizeof(double) * ne * nf);
    wmatrix(la, lb, lc, ld, Ra, Rb, Rc, Rd, na, ea, ca, nb, eb, cb, nc, ec, cc, nd, ed, cd, kappa, W);
    double AB[3] = {Ra[0] - Rb[0], Ra[1] - Rb[1], Ra[2] - Rb[2]};
    double CD[3] = {Rc[0] - Rd[0], Rc[1] - Rd[1], Rc[2] - Rd[2]};
    double *X = (double *)malloc(sizeof(double) * ne * Nc * Nd);   /* [e][cd] */
    for (int e = 0; e < ne; ++e) hrr_pair(lc, ld, CD, W + e * nf, X + (size_t)e * Nc * Nd);
    double *col = (double *)malloc(sizeof(double) * ne);
    double *res = (double *)malloc(sizeof(double) * Na * Nb);
    for (int q = 0; q < Nc * Nd; ++q) {
        for (int e = 0; e < ne; ++e) col[e] = X[(size_t)e * Nc * Nd + q];
        hrr_pair(la, lb, AB, col, res);
        for (int ab = 0; ab < Na * Nb; ++ab) G[ab + (size_t)Na * Nb * q] = res[ab];
    }
    free(W); free(X); free(col); free(res);
}

/* ---------------------------------------------------------------------- */
/* Two-centre Hermite form (no horizontal recurrence).                    */
/*                                                                        */
/* The W-matrix + HRR route above contracts (e0| on centre A over the     */
/* primitive pairs and then moves angular momentum to B with              */
/* (a,b| = sum_k C(b,k) (A-B)^{b-k} (a+k,0|.  For a primitive pair whose  */
/* product centre P lies near B (tight primitive on B, diffuse one on A)  */
/* that sum cancels ~ (|AB| sqrt(p))^{l_b}: for f shells contracted over  */
/* [0.05, 5e3] on atoms 4.6 bohr apart the (ff|ff) quartet loses every    */
/* digit (bra-ket symmetry broken by 33% of its largest element).  No     */
/* single orientation of a contracted pair avoids it when both shells mix */
/* tight and diffuse primitives.  The two-centre coefficients E^{ij}_t of */
/* (x-A)^i (x-B)^j exp(-p(x-P)^2) (McMurchie-Davidson; Helgaker 9.5.6)    */
/* are built per primitive pair from PA and PB without cancellation, and  */
/*   (ab|cd) = sum E^{ab}_{tuv} (-1)^{tau+nu+phi} E^{cd}_{tau nu phi}     */
/*             R_{t+tau,u+nu,v+phi}                                       */
/* is the same integral.  The CUDA library evaluates this form; the       */
/* W-matrix route stays here as the restatement of the reference.        */
/* ---------------------------------------------------------------------- */

/* offset of block (i, j), t = 0..i+j, in a per-axis table for i <= la, j major */
static inline int e2_off(int la, int i, int j)
{
    return (la + 1) * j * (j + 1) / 2 + j * la * (la + 1) / 2 + i * (j + 1) + i * (i - 1) / 2;
}
static inline int e2_size(int la, int lb) { return (la + 1) * (lb + 1) * (la + lb + 2) / 2; }

/* E^{ij}_t for i <= la, j <= lb (PA = P - A, PB = P - B along one axis) */
static void e2_coeffs(int la, int lb, double p, double PA, double PB, double *E)
{
    const double h = 1.0 / (2.0 * p);
    E[e2_off(la, 0, 0)] = 1.0;
    for (int i = 0; i < la; ++i) {
        const double *Ei = E + e2_off(la, i, 0);
        double *En = E + e2_off(la, i + 1, 0);
        for (int t = 0; t <= i + 1; ++t) {
            double v = 0.0;
            if (t >= 1) v += h * Ei[t - 1];
            if (t <= i) v += PA * Ei[t];
            if (t + 1 <= i) v += (t + 1) * Ei[t + 1];
            En[t] = v;
        }
    }
    for (int j = 0; j < lb; ++j)
        for (int i = 0; i <= la; ++i) {
            const double *Ej = E + e2_off(la, i, j);
            double *En = E + e2_off(la, i, j + 1);
            const int n = i + j;
            for (int t = 0; t <= n + 1; ++t) {
                double v = 0.0;
                if (t >= 1) v += h * Ej[t - 1];
                if (t <= n) v += PB * Ej[t];
                if (t + 1 <= n) v += (t + 1) * Ej[t + 1];
                En[t] = v;
            }
        }
}

static void cart_quartet_2c(int la, int lb, int lc, int ld,
                            const double *Ra, const double *Rb, const double *Rc, const double *Rd,
                            int na, const double *ea, const double *ca,
                            int nb, const double *eb, const double *cb,
                            int nc, const double *ec, const double *cc,
                            int nd, const double *ed, const double *cd,
                            double kappa, double *G)
{
    const int L1 = la + lb, L2 = lc + ld, LT = L1 + L2;
    const int Na = NCART(la), Nb = NCART(lb), Nc = NCART(lc), Nd = NCART(ld);
    const int a0 = CART_OFF(la), b0 = CART_OFF(lb), c0 = CART_OFF(lc), d0 = CART_OFF(ld);
    const int sab = e2_size(la, lb), scd = e2_size(lc, ld);
    memset(G, 0, sizeof(double) * (size_t)Na * Nb * Nc * Nd);
    double Rab2 = 0, Rcd2 = 0;
    for (int i = 0; i < 3; ++i) {
        Rab2 += (Ra[i] - Rb[i]) * (Ra[i] - Rb[i]);
        Rcd2 += (Rc[i] - Rd[i]) * (Rc[i] - Rd[i]);
    }
    double *Eab = (double *)malloc(sizeof(double) * 3 * sab);
    double *Ecd = (double *)malloc(sizeof(double) * 3 * scd);
    double *R = (double *)malloc(sizeof(double) * HERM_N(LT));
    double *S = (double *)malloc(sizeof(double) * HERM_N(L1));
    double F[MAXLT + 1];
    for (int gd = 0; gd < nd; ++gd)
        for (int gc = 0; gc < nc; ++gc) {
            const double Q = ec[gc] + ed[gd];
            const double mucd = ec[gc] * ed[gd] / Q;
            double Rq[3];
            for (int i = 0; i < 3; ++i) {
                Rq[i] = (ec[gc] * Rc[i] + ed[gd] * Rd[i]) / Q;
                e2_coeffs(lc, ld, Q, Rq[i] - Rc[i], Rq[i] - Rd[i], Ecd + i * scd);
            }
            for (int gb = 0; gb < nb; ++gb)
                for (int ga = 0; ga < na; ++ga) {
                    const double P = ea[ga] + eb[gb];
                    const double muab = ea[ga] * eb[gb] / P;
                    double Rp[3], Rpq[3];
                    for (int i = 0; i < 3; ++i) {
                        Rp[i] = (ea[ga] * Ra[i] + eb[gb] * Rb[i]) / P;
                        Rpq[i] = Rp[i] - Rq[i];
                        e2_coeffs(la, lb, P, Rp[i] - Ra[i], Rp[i] - Rb[i], Eab + i * sab);
                    }
                    const double kabcd = exp(-muab * Rab2 - mucd * Rcd2);
                    const double PQ = P * Q;
                    const double alpha = PQ / (P + Q + kappa * PQ);
                    const double N = 2.0 * pow(PI, 2.5) / (PQ * sqrt(P + Q + kappa * PQ));
                    const double e000 = N * ca[ga] * cb[gb] * cc[gc] * cd[gd] * kabcd;
                    const double T = alpha * (Rpq[0] * Rpq[0] + Rpq[1] * Rpq[1] + Rpq[2] * Rpq[2]);
                    orc_fm(LT, T, F);
                    rtuv(LT, F, alpha, Rpq[0], Rpq[1], Rpq[2], R);
                    for (int d = 0; d < Nd; ++d)
                        for (int c = 0; c < Nc; ++c) {
                            const int cx = g_cx[c0 + c], cy = g_cy[c0 + c], cz = g_cz[c0 + c];
                            const int dx = g_cx[d0 + d], dy = g_cy[d0 + d], dz = g_cz[d0 + d];
                            const double *Ex = Ecd + e2_off(lc, cx, dx);
                            const double *Ey = Ecd + scd + e2_off(lc, cy, dy);
                            const double *Ez = Ecd + 2 * scd + e2_off(lc, cz, dz);
                            /* S(h) = sum_g (-1)^|g| E^{cd}_g R(h + g), h up to level L1 */
                            for (int k = 0; k <= L1; ++k)
                                for (int s = 0; s <= k; ++s)
                                    for (int v = 0; v <= s; ++v) {
                                        const int u = s - v, t = k - s;
                                        double acc = 0.0;
                                        for (int p3 = 0; p3 <= cz + dz; ++p3)
                                            for (int p2 = 0; p2 <= cy + dy; ++p2)
                                                for (int p1 = 0; p1 <= cx + dx; ++p1) {
                                                    const double sg = ((p1 + p2 + p3) & 1) ? -1.0 : 1.0;
                                                    acc += sg * Ex[p1] * Ey[p2] * Ez[p3] *
                                                           R[herm_idx(t + p1, u + p2, v + p3)];
                                                }
                                        S[herm_idx(t, u, v)] = acc;
                                    }
                            const size_t q = (size_t)c + (size_t)Nc * d;
                            for (int bi = 0; bi < Nb; ++bi)
                                for (int ai = 0; ai < Na; ++ai) {
                                    const int ax = g_cx[a0 + ai], ay = g_cy[a0 + ai], az = g_cz[a0 + ai];
                                    const int bx = g_cx[b0 + bi], by = g_cy[b0 + bi], bz = g_cz[b0 + bi];
                                    const double *Fx = Eab + e2_off(la, ax, bx);
                                    const double *Fy = Eab + sab + e2_off(la, ay, by);
                                    const double *Fz = Eab + 2 * sab + e2_off(la, az, bz);
                                    double acc = 0.0;
                                    for (int v = 0; v <= az + bz; ++v)
                                        for (int u = 0; u <= ay + by; ++u)
                                            for (int t = 0; t <= ax + bx; ++t)
                                                acc += Fx[t] * Fy[u] * Fz[v] * S[herm_idx(t, u, v)];
                                    G[(size_t)ai + (size_t)Na * bi + (size_t)Na * Nb * q] += e000 * acc;
                                }
                        }
                }
        }
    free(Eab); free(Ecd); free(R); free(S);
}

/* Integral scheme of every quartet the oracle evaluates: 1 = two-centre
 * Hermite form (what the CUDA library computes, default), 0 = the
 * reference's W-matrix + HRR route. */
static int g_eri_scheme = 1;
void orc_set_eri_scheme(int scheme) { g_eri_scheme = scheme ? 1 : 0; }

static void cart_quartet_any(int la, int lb, int lc, int ld,
                             const double *Ra, const double *Rb, const double *Rc, const double *Rd,
                             int na, const double *ea, const double *ca,
                             int nb, const double *eb, const double *cb,
                             int nc, const double *ec, const double *cc,
                             int nd, const double *ed, const double *cd,
                             double kappa, double *G)
{
    if (g_eri_scheme)
        cart_quartet_2c(la, lb, lc, ld, Ra, Rb, Rc, Rd, na, ea, ca, nb, eb, cb, nc, ec, cc, nd, ed, cd, kappa, G);
    else
        cart_quartet(la, lb, lc, ld, Ra, Rb, Rc, Rd, na, ea, ca, nb, eb, cb, nc, ec, cc, nd, ed, cd, kappa, G);
}

/* Apply the per-shell transforms T (nfunc x ncart) to every index of a
 * 4-index block, a fastest (auto2e_SpherTransf.f90 + auto2e_Normalize_*). */
static void transform4(const double *G, int n[4], const double *T[4], int nf[4], double *out)
{
    /* successive one-index transforms; the current index is always the
     * slowest-varying after a rotation of the layout */
    size_t cap = 1;
    for (int i = 0; i < 4; ++i) cap *= (size_t)((n[i] > nf[i]) ? n[i] : nf[i]);
    double *a = (double *)malloc(sizeof(double) * cap);
    double *b = (double *)malloc(sizeof(double) * cap);
    int dims[4] = {n[0], n[1], n[2], n[3]};
    size_t tot = (size_t)dims[0] * dims[1] * dims[2] * dims[3];
    memcpy(a, G, sizeof(double) * tot);
    for (int idx = 0; idx < 4; ++idx) {
        /* a is laid out with index 0 fastest: dims[0..3]; transform index 0
         * and move it to the slowest position */
        int d0 = dims[0];
        size_t rest = tot / d0;
        int m0 = nf[idx];
        for (size_t r = 0; r < rest; ++r)
            for (int m = 0; m < m0; ++m) {
                double s = 0.0;
                for (int c = 0; c < d0; ++c) s += T[idx][m * d0 + c] * a[c + (size_t)d0 * r];
                b[r + rest * m] = s;
            }
        dims[0] = dims[1]; dims[1] = dims[2]; dims[2] = dims[3]; dims[3] = m0;
        tot = rest * m0;
        double *t = a; a = b; b = t;
    }
    memcpy(out, a, sizeof(double) * tot);
    free(a); free(b);
}

static inline int nfunc(const orc_basis *b, int s)
{
    return b->spher ? 2 * b->L[s] + 1 : NCART(b->L[s]);
}

/* One normalised (spherical or Cartesian) shell quartet, V(a,b,c,d) with a
 * fastest -- the layout a caller of Auto2eERI obtains by passing the shells
 * in the order (D,C,B,A) (auto2e.f90:1-34, TwoStepCholesky_Step1.f90:812-838). */
/* Canonical orientation of a class, as the reference's frontends arrange it
 * (e.g. auto2e_frontend_1_2_1_2, auto2e_eri_dpdp.f90:334-351): the higher
 * angular momentum first within each pair, and the bra pair not below the
 * ket pair in the (l_hi, l_lo) order.  The HRR's rounding depends on the
 * orientation, so the oracle evaluates the same canonical class. */
static inline int pair_rank(int lhi, int llo) { return lhi * (lhi + 1) / 2 + llo; }

static double min_exponent(const orc_basis *b, int s)
{
    double m = 1e300;
    for (int i = 0; i < b->nprim[s]; ++i) m = fmin(m, b->exps[b->prim_off[s] + i]);
    return m;
}

/* 1 if shell x stays first in the pair (x, y).  Higher l first, as in the
 * reference.  For equal l the reference keeps the given order; here the
 * shell with the larger smallest exponent goes first, because the HRR
 * (a,b| = sum C(b,k) (A-B)^{b-k} (a+k,0| loses up to ~6 digits when A is the
 * diffuse shell of a distant pair (the product centre P is then far from A).
 * Ties keep the given order. */
static int orient_first(const orc_basis *b, int x, int y)
{
    if (b->L[x] != b->L[y]) return b->L[x] > b->L[y];
    return min_exponent(b, x) >= min_exponent(b, y);
}

int orc_eri_quartet(const orc_basis *b, int A, int B, int C, int D, double kappa, double *out)
{
    int sh[4] = {A, B, C, D};
    int l[4], n[4], nf[4];
    const double *T[4];
    for (int i = 0; i < 4; ++i) {
        l[i] = b->L[sh[i]];
        if (l[i] > ORC_MAXL) return -1;
        n[i] = NCART(l[i]);
        nf[i] = nfunc(b, sh[i]);
        T[i] = b->T + b->T_off[sh[i]];
    }
    /* position of each canonical index in the requested order; within a pair
     * of equal l the tighter shell (larger smallest exponent) is the origin
     * of the horizontal recurrence (see orient_first) */
    int pos[4] = {0, 1, 2, 3};
    if (!orient_first(b, A, B)) { pos[0] = 1; pos[1] = 0; }
    if (!orient_first(b, C, D)) { pos[2] = 3; pos[3] = 2; }
    if (pair_rank(l[pos[0]], l[pos[1]]) < pair_rank(l[pos[2]], l[pos[3]])) {
        int t0 = pos[0], t1 = pos[1];
        pos[0] = pos[2]; pos[1] = pos[3]; pos[2] = t0; pos[3] = t1;
    }
    int cs[4], cl[4], cn[4];
    for (int i = 0; i < 4; ++i) { cs[i] = sh[pos[i]]; cl[i] = l[pos[i]]; cn[i] = n[pos[i]]; }
    size_t tot = (size_t)n[0] * n[1] * n[2] * n[3];
    double *Gc = (double *)malloc(sizeof(double) * tot);
    double *G = (double *)malloc(sizeof(double) * tot);
    cart_quartet_any(cl[0], cl[1], cl[2], cl[3],
                 b->coords + 3 * cs[0], b->coords + 3 * cs[1], b->coords + 3 * cs[2], b->coords + 3 * cs[3],
                 b->nprim[cs[0]], b->exps + b->prim_off[cs[0]], b->coefs + b->prim_off[cs[0]],
                 b->nprim[cs[1]], b->exps + b->prim_off[cs[1]], b->coefs + b->prim_off[cs[1]],
                 b->nprim[cs[2]], b->exps + b->prim_off[cs[2]], b->coefs + b->prim_off[cs[2]],
                 b->nprim[cs[3]], b->exps + b->prim_off[cs[3]], b->coefs + b->prim_off[cs[3]],
                 kappa, Gc);
    /* back to the requested order (index 0 fastest) */
    size_t cstr[4] = {1, (size_t)cn[0], (size_t)cn[0] * cn[1], (size_t)cn[0] * cn[1] * cn[2]};
    size_t str_of_orig[4];
    for (int i = 0; i < 4; ++i) str_of_orig[pos[i]] = cstr[i];
    for (size_t idx = 0; idx < tot; ++idx) {
        size_t r = idx, off = 0;
        for (int i = 0; i < 4; ++i) { off += (r % n[i]) * str_of_orig[i]; r /= n[i]; }
        G[idx] = Gc[off];
    }
    transform4(G, n, T, nf, out);
    free(G); free(Gc);
    return 0;
}

/* ====================================================================== */
/* SLATEC DSORT (Singleton quicksort, carry DY), sort.f90:19-... (kflag=+-2). */
/* The published SLATEC algorithm, restated with 0-based arrays.           */
/* ====================================================================== */
static void dsort0(double *dx, int64_t *dy, int64_t n, int kflag)
{
    if (n <= 1) return;
    if (kflag <= -1) for (int64_t i = 0; i < n; ++i) dx[i] = -dx[i];
    /* 1-based views */
    double *X = dx - 1;
    int64_t *Y = dy - 1;
    int64_t il[21], iu[21];
    int64_t m = 1, i = 1, j = n, k, l, ij;
    double r = 0.375, t, tt;
    int64_t ty, tty;
L110:
    if (i == j) goto L150;
    if (r <= 0.5898437) r += 3.90625e-2; else r -= 0.21875;
L120:
    k = i;
    ij = i + (int64_t)((j - i) * r);
    t = X[ij]; ty = Y[ij];
    if (X[i] > t) { X[ij] = X[i]; X[i] = t; t = X[ij]; Y[ij] = Y[i]; Y[i] = ty; ty = Y[ij]; }
    l = j;
    if (X[j] < t) {
        X[ij] = X[j]; X[j] = t; t = X[ij]; Y[ij] = Y[j]; Y[j] = ty; ty = Y[ij];
        if (X[i] > t) { X[ij] = X[i]; X[i] = t; t = X[ij]; Y[ij] = Y[i]; Y[i] = ty; ty = Y[ij]; }
    }
L130:
    l = l - 1;
    if (X[l] > t) goto L130;
L140:
    k = k + 1;
    if (X[k] < t) goto L140;
    if (k <= l) {
        tt = X[l]; X[l] = X[k]; X[k] = tt;
        tty = Y[l]; Y[l] = Y[k]; Y[k] = tty;
        goto L130;
    }
    if (l - i > j - k) { il[m - 1] = i; iu[m - 1] = l; i = k; m = m + 1; }
    else { il[m - 1] = k; iu[m - 1] = j; j = l; m = m + 1; }
    goto L160;
L150:
    m = m - 1;
    if (m == 0) goto L190;
    i = il[m - 1]; j = iu[m - 1];
L160:
    if (j - i >= 1) goto L120;
    if (i == 1) goto L110;
    i = i - 1;
L170:
    i = i + 1;
    if (i == j) goto L150;
    t = X[i + 1]; ty = Y[i + 1];
    if (X[i] <= t) goto L170;
    k = i;
L180:
    X[k + 1] = X[k]; Y[k + 1] = Y[k];
    k = k - 1;
    if (t < X[k]) goto L180;
    X[k + 1] = t; Y[k + 1] = ty;
    goto L170;
L190:
    if (kflag <= -1) for (int64_t q = 0; q < n; ++q) dx[q] = -dx[q];
}

/* ====================================================================== */
/* Work counters (same layout as the library's gci_stats): [0..4] GEMM      */
/* flops of M - L L^T, new vectors, potrf+trtri, Inv_L product, AO->MO;    */
/* [5..7] shell quartets, primitive quartets, integrals; then per class    */
/* (bra pair type, ket pair type) the same three counts.                   */
/* ====================================================================== */
#define NPT 21   /* pair types for l <= 5 */
static double g_stats[8 + 3 * NPT * NPT];

static inline int ptype(int la, int lb)
{
    int hi = la > lb ? la : lb, lo = la > lb ? lb : la;
    return hi * (hi + 1) / 2 + lo;
}

void orc_stats_reset(void) { memset(g_stats, 0, sizeof(g_stats)); }

void orc_stats(double *out, int n)
{
    for (int i = 0; i < n && i < (int)(sizeof(g_stats) / sizeof(double)); ++i) out[i] = g_stats[i];
}

static void count_quartet(const orc_basis *b, int A, int B, int C, int D)
{
    int t1 = ptype(b->L[A], b->L[B]), t2 = ptype(b->L[C], b->L[D]);
    int hi = t1 > t2 ? t1 : t2, lo = t1 > t2 ? t2 : t1;
    double nf = (double)nfunc(b, A) * nfunc(b, B) * nfunc(b, C) * nfunc(b, D);
    double np = (double)b->nprim[A] * b->nprim[B] * b->nprim[C] * b->nprim[D];
    double *c = g_stats + 8 + 3 * (hi * NPT + lo);
#pragma omp atomic
    c[0] += 1.0;
#pragma omp atomic
    c[1] += np;
#pragma omp atomic
    c[2] += nf;
#pragma omp atomic
    g_stats[5] += 1.0;
#pragma omp atomic
    g_stats[6] += np;
#pragma omp atomic
    g_stats[7] += nf;
}

/* ====================================================================== */
/* Two-step Cholesky                                                        */
/* ====================================================================== */

/* chol2_pq2p_ge_q, TwoStepCholesky_Step2.f90:422-466 (1-based in and out) */
static void pq2p_ge_q(int64_t pq, int64_t n, int64_t *p, int64_t *q)
{
    int64_t q_base = (pq - 1) / (n + 1) + 1;
    int64_t v = pq - (n + 1) * (q_base - 1);
    int64_t interval1 = n - q_base + 1;
    int64_t in2 = v / (interval1 + 1);
    int64_t in1 = in2 ^ 1;
    *p = in1 * (q_base + v - 1) + in2 * (v - interval1 + n - q_base);
    *q = in1 * q_base + in2 * interval1;
}

/* ERI block of shells (A,B,C,D), a fastest; scratch is caller's */
static void quartet_into(const orc_basis *b, int A, int B, int C, int D, double kappa, double *V)
{
    count_quartet(b, A, B, C, D);
    orc_eri_quartet(b, A, B, C, D, kappa, V);
}

/* Pair-local orbital-pair index for (a,b) in shell pair (A,B): a + Na b when
 * A != B; column-wise lower triangle (b outer, a = b..Na) when A == B
 * (chol2_write_Vdiag / _Vaacd / _Vaacc, Step1.f90:100-199).  -1 if a < b. */
static inline int64_t pair_local(int a, int bb, int Na, int same)
{
    if (!same) return a + (int64_t)Na * bb;
    if (a < bb) return -1;
    return (int64_t)bb * Na - (int64_t)bb * (bb - 1) / 2 + (a - bb);
}

int orc_cholesky(const orc_basis *b, double tau, double kappa, int max_block_dim,
                 int want_rkpq, int pivot_decode_storage, int nthreads, orc_chol *res)
{
    return orc_cholesky_forced(b, tau, kappa, max_block_dim, want_rkpq, pivot_decode_storage, nthreads,
                               NULL, 0, 0, res);
}

int orc_cholesky_forced(const orc_basis *b, double tau, double kappa, int max_block_dim,
                        int want_rkpq, int pivot_decode_storage, int nthreads,
                        const int64_t *forced_order, int64_t nforced, int stage_limit, orc_chol *res)
{
    memset(res, 0, sizeof(*res));
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    int nsh = b->nshells;
    int lmax = 0;
    int64_t nao = 0;
    for (int s = 0; s < nsh; ++s) { if (b->L[s] > lmax) lmax = b->L[s]; nao += nfunc(b, s); }
    if (lmax > ORC_MAXL) return -1;
    if (orc_boys_init(4 * ORC_MAXL) != 0) return -2;
    int maxnang = b->spher ? 2 * lmax + 1 : NCART(lmax);
    int64_t maxnsp = (int64_t)nsh * (nsh + 1) / 2;
    int64_t maxnorb = nao * (nao + 1) / 2;
    res->nao = nao;

    /* ---------------- chol2_Vdiag, Step1.f90:202-279 ---------------- */
    double *Vdiag = (double *)malloc(sizeof(double) * maxnorb);
    int64_t *vdloc = (int64_t *)malloc(sizeof(int64_t) * maxnsp);
    int *vddim = (int *)malloc(sizeof(int) * maxnsp);
    int *vdpair = (int *)malloc(sizeof(int) * 2 * maxnsp);
    {
        int64_t loc = 0, sp = 0;
        for (int B = 0; B < nsh; ++B)
            for (int A = B; A < nsh; ++A) {
                int Na = nfunc(b, A), Nb = nfunc(b, B);
                int dim = (A != B) ? Na * Nb : Na * (Na + 1) / 2;
                vdloc[sp] = loc; vddim[sp] = dim; vdpair[2 * sp] = A; vdpair[2 * sp + 1] = B;
                loc += dim; ++sp;
            }
    }
#pragma omp parallel for schedule(dynamic)
    for (int64_t sp = 0; sp < maxnsp; ++sp) {
        int A = vdpair[2 * sp], B = vdpair[2 * sp + 1];
        int Na = nfunc(b, A), Nb = nfunc(b, B);
        double *V = (double *)malloc(sizeof(double) * (size_t)Na * Nb * Na * Nb);
        quartet_into(b, A, B, A, B, kappa, V);
        int64_t p = vdloc[sp];
        for (int bb = 0; bb < Nb; ++bb)
            for (int a = (A == B) ? bb : 0; a < Na; ++a)
                Vdiag[p++] = V[a + (size_t)Na * (bb + (size_t)Nb * (a + (size_t)Na * bb))];
        free(V);
    }

    /* ---------------- chol2_DefineBase, Step1.f90:282-442 ---------------- */
    double *vdmax = (double *)malloc(sizeof(double) * maxnsp);
    int64_t *idxmap = (int64_t *)malloc(sizeof(int64_t) * maxnsp);
    double maxdrs = -1e300;
    for (int64_t sp = 0; sp < maxnsp; ++sp) {
        double m = -1e300;
        for (int i = 0; i < vddim[sp]; ++i) if (Vdiag[vdloc[sp] + i] > m) m = Vdiag[vdloc[sp] + i];
        vdmax[sp] = m; idxmap[sp] = sp;
        if (m > maxdrs) maxdrs = m;
    }
    if (!(maxdrs > 0.0)) return -3;
    double thr = fmin(tau, 1.0e-8);
    double prescreen = thr * thr / maxdrs;
    dsort0(vdmax, idxmap, maxnsp, 2);
    double discarded = 0.0;
    int64_t k0 = 1, k1 = maxnsp;   /* 1-based, as in the reference */
    for (int64_t k = 1; k <= maxnsp; ++k) {
        int64_t sp = idxmap[k - 1];
        double sum = 0.0, mx = -1e300;
        for (int i = 0; i < vddim[sp]; ++i) {
            sum += Vdiag[vdloc[sp] + i];
            if (Vdiag[vdloc[sp] + i] > mx) mx = Vdiag[vdloc[sp] + i];
        }
        if (mx <= prescreen) { discarded += sum; k0 = k; }   /* keeps k0 on the last discarded pair */
        else break;
    }
    res->trace_error = discarded;
    int64_t nsp = k1 - k0 + 1;
    res->nshellpairs = nsp;
    res->shellpairs = (int *)malloc(sizeof(int) * 2 * nsp);
    res->shellpairloc = (int64_t *)malloc(sizeof(int64_t) * 3 * nsp);
    res->shellpairdim = (int *)malloc(sizeof(int) * nsp);
    int64_t npq = 0;
    for (int64_t k = k0; k <= k1; ++k) npq += vddim[idxmap[k - 1]];
    res->norbpairs = npq;
    double *D = (double *)malloc(sizeof(double) * npq);
    {
        int64_t p = 0;
        for (int64_t k = k0, s = 0; k <= k1; ++k, ++s) {
            int64_t l = idxmap[k - 1];
            res->shellpairs[2 * s] = vdpair[2 * l];
            res->shellpairs[2 * s + 1] = vdpair[2 * l + 1];
            res->shellpairdim[s] = vddim[l];
            res->shellpairloc[3 * s + 0] = p;
            memcpy(D + p, Vdiag + vdloc[l], sizeof(double) * vddim[l]);
            p += vddim[l];
        }
    }
    free(vdmax); free(idxmap); free(Vdiag); free(vdloc); free(vddim); free(vdpair);

    /* ---------------- chol2_DefineSubsets / DivideOrbPairs, :445-530 ---------------- */
    {
        int64_t ns = (npq + max_block_dim - 1) / max_block_dim;
        if (ns < 1) ns = 1;
        res->nsubsets = ns;
        res->subsetdim = (int64_t *)calloc(ns, sizeof(int64_t));
        res->subsetbounds = (int64_t *)malloc(sizeof(int64_t) * 2 * ns);
        int64_t target = (npq + ns - 1) / ns;
        for (int64_t k = 1; k <= ns; ++k) {
            int64_t lo, hi;   /* 1-based shell pair bounds, 0 = empty */
            if (k == 1) lo = 1;
            else {
                int64_t prev = res->subsetbounds[2 * (k - 2) + 1] + 1;   /* stored 0-based */
                lo = (prev < nsp && prev > 0) ? prev + 1 : 0;
            }
            int64_t dim = 0;
            hi = lo;
            if (lo > 0) {
                if (k < ns) {
                    int64_t berr[2] = {npq, npq}, bloc[2] = {lo, lo};
                    for (int64_t s = lo; s <= nsp; ++s) {
                        res->shellpairloc[3 * (s - 1) + 1] = dim;
                        res->shellpairloc[3 * (s - 1) + 2] = k - 1;
                        dim += res->shellpairdim[s - 1];
                        if (dim >= target) { bloc[1] = s; berr[1] = dim - target; break; }
                        else { bloc[0] = s; berr[0] = dim - target; }
                    }
                    if (llabs(berr[0]) < llabs(berr[1])) { hi = bloc[0]; dim = berr[0] + target; }
                    else { hi = bloc[1]; dim = berr[1] + target; }
                } else {
                    hi = nsp;
                    for (int64_t s = lo; s <= hi; ++s) {
                        res->shellpairloc[3 * (s - 1) + 1] = dim;
                        res->shellpairloc[3 * (s - 1) + 2] = k - 1;
                        dim += res->shellpairdim[s - 1];
                    }
                }
            }
            res->subsetdim[k - 1] = dim;
            res->subsetbounds[2 * (k - 1)] = lo - 1;
            res->subsetbounds[2 * (k - 1) + 1] = hi - 1;
        }
        int64_t mx = 0;
        for (int64_t k = 0; k < ns; ++k) if (res->subsetdim[k] > mx) mx = res->subsetdim[k];
        res->max_subset_dim = mx;
    }

    if (stage_limit == 1) { free(D); return 1; }
    /* ---------------- chol2_Pivots, Step1.f90:884-1103 ---------------- */
    int64_t maxnchol = (int64_t)ceil(nao * 15.0);
    if (maxnchol > npq) maxnchol = npq;
    res->pivots = (int *)calloc(npq, sizeof(int));
    res->pivot_order = (int64_t *)malloc(sizeof(int64_t) * (maxnchol > 0 ? maxnchol : 1));
    res->pivot_dmax = (double *)malloc(sizeof(double) * (maxnchol > 0 ? maxnchol : 1));
    int64_t *candmap = (int64_t *)malloc(sizeof(int64_t) * nsp);  /* shell pair ids */
    int64_t *compr = (int64_t *)malloc(sizeof(int64_t) * nsp);    /* compressed loc per pair */
    int64_t ncand_sp = nsp, ncand = npq;
    for (int64_t s = 0; s < nsp; ++s) { candmap[s] = s; compr[s] = res->shellpairloc[3 * s]; }
    /* stored vectors: Lst[j * ldl + pq] for compressed pq, j < nchol */
    int64_t ldl = npq;
    double *Lst = (double *)malloc(sizeof(double) * (size_t)ldl * (maxnchol > 0 ? maxnchol : 1));
    int64_t nchol = 0;
    double dmax = -1e300;
    for (int64_t p = 0; p < npq; ++p) if (D[p] > dmax) dmax = D[p];
    int converged = 0;
    int macro_go = (maxnchol > 0) && (forced_order == NULL);
    if (forced_order) {
        /* step 2 on a given pivot sequence (FULL indices, 0-based) */
        for (int64_t j = 0; j < nforced; ++j) {
            res->pivots[forced_order[j]] = 1;
            res->pivot_order[j] = forced_order[j];
            res->pivot_dmax[j] = 0.0;
        }
        nchol = nforced;
        converged = 1;
    }
    int64_t nmacro = 0;
    int64_t *bmap = (int64_t *)malloc(sizeof(int64_t) * nsp);
    int64_t *colloc = (int64_t *)malloc(sizeof(int64_t) * nsp);
    double *sortv = (double *)malloc(sizeof(double) * nsp);
    int64_t *sorti = (int64_t *)malloc(sizeof(int64_t) * nsp);
    int64_t nbatch = 0, nbatch_sp = 0;
    while (macro_go) {
        ++nmacro;
        /* chol2_DefineCandidates :533-575 */
        for (int64_t k = 0; k < ncand_sp; ++k) {
            int64_t s = candmap[k];
            double m = -1e300;
            for (int i = 0; i < res->shellpairdim[s]; ++i)
                if (D[compr[s] + i] > m) m = D[compr[s] + i];
            sortv[k] = m; sorti[k] = s;
        }
        dsort0(sortv, sorti, ncand_sp, -2);
        int64_t old = ncand_sp;
        ncand_sp = 0; int64_t ncand_new = 0;
        int64_t *newcand = (int64_t *)malloc(sizeof(int64_t) * (old > 0 ? old : 1));
        for (int64_t k = 0; k < old; ++k) {
            if (sortv[k] > tau) { newcand[ncand_sp++] = sorti[k]; ncand_new += res->shellpairdim[sorti[k]]; }
            else break;
        }
        /* chol2_Compress :16-97 */
        {
            double *Dn = (double *)malloc(sizeof(double) * (ncand_new > 0 ? ncand_new : 1));
            int64_t *newloc = (int64_t *)malloc(sizeof(int64_t) * (ncand_sp > 0 ? ncand_sp : 1));
            int64_t pos = 0;
            for (int64_t g = 0; g < ncand_sp; ++g) {
                int64_t s = newcand[g];
                newloc[g] = pos;
                memcpy(Dn + pos, D + compr[s], sizeof(double) * res->shellpairdim[s]);
                pos += res->shellpairdim[s];
            }
            if (nchol > 0) {
                double *Ln = (double *)malloc(sizeof(double) * (size_t)(ncand_new > 0 ? ncand_new : 1) * maxnchol);
#pragma omp parallel for
                for (int64_t j = 0; j < nchol; ++j)
                    for (int64_t g = 0; g < ncand_sp; ++g) {
                        int64_t s = newcand[g];
                        memcpy(Ln + j * ncand_new + newloc[g], Lst + j * ldl + compr[s],
                               sizeof(double) * res->shellpairdim[s]);
                    }
                free(Lst); Lst = Ln;
            }
            ldl = ncand_new;
            for (int64_t g = 0; g < ncand_sp; ++g) compr[newcand[g]] = newloc[g];
            free(D); D = Dn;
            free(newloc);
        }
        memcpy(candmap, newcand, sizeof(int64_t) * ncand_sp);
        free(newcand);
        ncand = ncand_new;
        int64_t maxnbatch = maxnang * maxnang > 1000 ? maxnang * maxnang : 1000;
        if (maxnbatch > ncand) maxnbatch = ncand;
        double dmin = fmax(0.01 * dmax, tau);
        /* chol2_DefineBatch :578-625 */
        for (int64_t k = 0; k < ncand_sp; ++k) {
            int64_t s = candmap[k];
            double m = -1e300;
            for (int i = 0; i < res->shellpairdim[s]; ++i)
                if (D[compr[s] + i] > m) m = D[compr[s] + i];
            sortv[k] = m; sorti[k] = s;
        }
        dsort0(sortv, sorti, ncand_sp, -2);
        nbatch_sp = 0; nbatch = 0;
        for (int64_t k = 0; k < ncand_sp; ++k) {
            int64_t s = sorti[k];
            int dim = res->shellpairdim[s];
            if (sortv[k] > dmin && nbatch + dim <= maxnbatch) {
                colloc[k] = nbatch; bmap[k] = s; nbatch_sp = k + 1; nbatch += dim;
            } else break;
        }
        /* chol2_M :733-856 -- M(ncand x nbatch), column-major */
        double *M = (double *)calloc((size_t)(ncand > 0 ? ncand : 1) * (nbatch > 0 ? nbatch : 1), sizeof(double));
#pragma omp parallel for collapse(2) schedule(dynamic)
        for (int64_t L = 0; L < nbatch_sp; ++L)
            for (int64_t K = 0; K < ncand_sp; ++K) {
                int64_t sab = candmap[K], scd = bmap[L];
                int A = res->shellpairs[2 * sab], B = res->shellpairs[2 * sab + 1];
                int C = res->shellpairs[2 * scd], Dd = res->shellpairs[2 * scd + 1];
                int Na = nfunc(b, A), Nb = nfunc(b, B), Nc = nfunc(b, C), Nd = nfunc(b, Dd);
                double *V = (double *)malloc(sizeof(double) * (size_t)Na * Nb * Nc * Nd);
                quartet_into(b, A, B, C, Dd, kappa, V);
                int64_t p0 = compr[sab], q0 = colloc[L];
                for (int d = 0; d < Nd; ++d)
                    for (int c = 0; c < Nc; ++c) {
                        int64_t cl = pair_local(c, d, Nc, C == Dd);
                        if (cl < 0) continue;
                        for (int bb = 0; bb < Nb; ++bb)
                            for (int a = 0; a < Na; ++a) {
                                int64_t al = pair_local(a, bb, Na, A == B);
                                if (al < 0) continue;
                                M[(p0 + al) + (size_t)ncand * (q0 + cl)] =
                                    V[a + (size_t)Na * (bb + (size_t)Nb * (c + (size_t)Nc * d))];
                            }
                    }
                free(V);
            }
        /* chol2_SubtractR :628-691 (M -= sum_j L_j(cand) L_j(batch)) */
        if (nchol > 0) {
            int64_t *brow = (int64_t *)malloc(sizeof(int64_t) * (nbatch > 0 ? nbatch : 1));
            for (int64_t k = 0; k < nbatch_sp; ++k) {
                int64_t s = bmap[k];
                for (int i = 0; i < res->shellpairdim[s]; ++i) brow[colloc[k] + i] = compr[s] + i;
            }
            g_stats[0] += 2.0 * ncand * nbatch * nchol;
#pragma omp parallel for schedule(static)
            for (int64_t q = 0; q < nbatch; ++q) {
                double *Mc = M + (size_t)ncand * q;
                for (int64_t j = 0; j < nchol; ++j) {
                    const double *Lj = Lst + j * ldl;
                    double f = Lj[brow[q]];
                    for (int64_t p = 0; p < ncand; ++p) Mc[p] -= Lj[p] * f;
                }
            }
            free(brow);
        }
        /* chol2_BatchMax :694-730 */
#define BATCHMAX()                                                                      \
        do {                                                                            \
            maxdpq = -1.0;                                                              \
            for (int64_t k = 0; k < nbatch_sp; ++k) {                                   \
                int64_t s = bmap[k];                                                    \
                for (int p = 0; p < res->shellpairdim[s]; ++p) {                        \
                    double dpq = D[compr[s] + p];                                       \
                    if (dpq > maxdpq) {                                                 \
                        maxdpq = dpq; maxloc = compr[s] + p;                            \
                        maxlocfull = res->shellpairloc[3 * s] + p;                      \
                        maxlocbatch = colloc[k] + p;                                    \
                    }                                                                   \
                }                                                                       \
            }                                                                           \
        } while (0)
        double maxdpq; int64_t maxloc = 0, maxlocfull = 0, maxlocbatch = 0;
        BATCHMAX();
        /* micro iterations :1030-1064 */
        double *Lm = (double *)malloc(sizeof(double) * (size_t)(ncand > 0 ? ncand : 1) * (nbatch > 0 ? nbatch : 1));
        int64_t j = 0;
        int micro = (nchol < maxnchol && nbatch > 0);
        while (micro) {
            ++j;
            res->pivots[maxlocfull] = 1;
            res->pivot_order[nchol] = maxlocfull;
            res->pivot_dmax[nchol] = maxdpq;
            ++nchol;
            /* chol2_Lj :859-881 */
            double *Lj = Lm + (size_t)ncand * (j - 1);
            memcpy(Lj, M + (size_t)ncand * maxlocbatch, sizeof(double) * ncand);
            g_stats[1] += 2.0 * ncand * (j - 1);
            if (j > 1) {
                double *Tq = (double *)malloc(sizeof(double) * (j - 1));
                for (int64_t i = 0; i < j - 1; ++i) Tq[i] = Lm[(size_t)ncand * i + maxloc];
#pragma omp parallel for schedule(static)
                for (int64_t p = 0; p < ncand; ++p) {
                    double s = 0.0;
                    for (int64_t i = 0; i < j - 1; ++i) s += Lm[(size_t)ncand * i + p] * Tq[i];
                    Lj[p] -= s;
                }
                free(Tq);
            }
            double sq = sqrt(maxdpq);
            for (int64_t p = 0; p < ncand; ++p) Lj[p] /= sq;
            memcpy(Lst + (nchol - 1) * ldl, Lj, sizeof(double) * ncand);
            for (int64_t p = 0; p < ncand; ++p) D[p] -= Lj[p] * Lj[p];
            BATCHMAX();
            if (maxdpq <= dmin) micro = 0;
            if (j == nbatch || nchol == maxnchol) micro = 0;
        }
#undef BATCHMAX
        free(Lm); free(M);
        dmax = -1e300;
        for (int64_t p = 0; p < ncand; ++p) if (D[p] > dmax) dmax = D[p];
        if (dmax <= tau) { converged = 1; macro_go = 0; }
        if (nchol == maxnchol || nbatch == 0) macro_go = 0;
        if (stage_limit == 2) macro_go = 0;
    }
    res->n_macro = nmacro;
    res->nvecs = nchol;
    res->converged = converged;
    res->dmax_final = dmax;
    free(bmap); free(colloc); free(sortv); free(sorti); free(candmap); free(compr);
    free(Lst); free(D);
    if (stage_limit == 2) { res->nvecs = nchol; return 2; }
    if (nchol == maxnchol && !converged) return -4;

    /* ---------------- chol2_PivotShellPairs, Step2.f90:469-534 ---------------- */
    res->pivshellpairs = (int *)malloc(sizeof(int) * nsp);
    res->pivshellpairloc = (int64_t *)malloc(sizeof(int64_t) * nsp);
    res->pivshellpairdim = (int *)malloc(sizeof(int) * nsp);
    res->pivorbpairs = (int *)malloc(sizeof(int) * (nchol > 0 ? nchol : 1));
    int64_t npsp = 0, q = 0;
    for (int64_t s = 0; s < nsp; ++s) {
        int A = res->shellpairs[2 * s], B = res->shellpairs[2 * s + 1];
        int64_t p0 = res->shellpairloc[3 * s];
        int dim = res->shellpairdim[s];
        int cnt = 0;
        for (int i = 0; i < dim; ++i) cnt += res->pivots[p0 + i];
        if (cnt == 0) continue;
        res->pivshellpairs[npsp] = (int)s;
        res->pivshellpairloc[npsp] = q;
        res->pivshellpairdim[npsp] = cnt;
        ++npsp;
        int Na = nfunc(b, A);
        for (int i = 0; i < dim; ++i) {
            if (!res->pivots[p0 + i]) continue;
            if (A != B) res->pivorbpairs[q] = i;
            else if (pivot_decode_storage) {
                /* column-wise triangle, the order Step 1 stores the pairs in */
                int bb = 0, rem = i;
                while (rem >= Na - bb) { rem -= Na - bb; ++bb; }
                res->pivorbpairs[q] = (bb + rem) + Na * bb;
            } else {
                int64_t pa, pb;
                pq2p_ge_q(i + 1, Na, &pa, &pb);
                res->pivorbpairs[q] = (int)((pa - 1) + Na * (pb - 1));
            }
            ++q;
        }
    }
    res->npivshellpairs = npsp;

    /* ---------------- chol2_Vpqrs, Step2.f90:76-187 ---------------- */
    int64_t N = nchol;
    double *V = (double *)calloc((size_t)(N > 0 ? N : 1) * (N > 0 ? N : 1), sizeof(double));
    int64_t ntri = npsp * (npsp + 1) / 2;
#pragma omp parallel for schedule(dynamic)
    for (int64_t kl = 1; kl <= ntri; ++kl) {
        int64_t K, L;
        pq2p_ge_q(kl, npsp, &K, &L);
        int64_t sab = res->pivshellpairs[K - 1], scd = res->pivshellpairs[L - 1];
        int A = res->shellpairs[2 * sab], B = res->shellpairs[2 * sab + 1];
        int C = res->shellpairs[2 * scd], Dd = res->shellpairs[2 * scd + 1];
        int Na = nfunc(b, A), Nb = nfunc(b, B);
        int Nc = nfunc(b, C), Nd = nfunc(b, Dd);
        double *Vq = (double *)malloc(sizeof(double) * (size_t)Na * Nb * Nc * Nd);
        quartet_into(b, A, B, C, Dd, kappa, Vq);
        int64_t pq0 = res->pivshellpairloc[K - 1], rs0 = res->pivshellpairloc[L - 1];
        for (int rs = 0; rs < res->pivshellpairdim[L - 1]; ++rs)
            for (int pq = 0; pq < res->pivshellpairdim[K - 1]; ++pq)
                V[(pq0 + pq) + (size_t)N * (rs0 + rs)] =
                    Vq[res->pivorbpairs[pq0 + pq] + (size_t)Na * Nb * res->pivorbpairs[rs0 + rs]];
        free(Vq);
    }
    g_stats[2] += 2.0 * (double)N * N * N / 3.0;
    /* real_Cholesky (dpotrf "L", upper zeroed) real_linalg.f90:39-58 */
    for (int64_t jj = 0; jj < N; ++jj) {
        double s = V[jj + N * jj];
        for (int64_t k = 0; k < jj; ++k) s -= V[jj + N * k] * V[jj + N * k];
        if (!(s > 0.0)) { free(V); return -5; }
        double d = sqrt(s);
        V[jj + N * jj] = d;
#pragma omp parallel for schedule(static)
        for (int64_t i = jj + 1; i < N; ++i) {
            double t = V[i + N * jj];
            for (int64_t k = 0; k < jj; ++k) t -= V[i + N * k] * V[jj + N * k];
            V[i + N * jj] = t / d;
        }
    }
    for (int64_t jj = 0; jj < N; ++jj) for (int64_t i = 0; i < jj; ++i) V[i + N * jj] = 0.0;
    /* real_LowerTriangularInverse (dtrtri "L","N") real_linalg.f90:60-72 */
    {
        double *Inv = (double *)calloc((size_t)(N > 0 ? N : 1) * (N > 0 ? N : 1), sizeof(double));
#pragma omp parallel for schedule(dynamic)
        for (int64_t c = 0; c < N; ++c) {
            Inv[c + N * c] = 1.0 / V[c + N * c];
            for (int64_t i = c + 1; i < N; ++i) {
                double s = 0.0;
                for (int64_t k = c; k < i; ++k) s += V[i + N * k] * Inv[k + N * c];
                Inv[i + N * c] = -s / V[i + N * i];
            }
        }
        free(V);
        res->inv_l = Inv;
    }

    /* ---------------- full-dimension vectors, TwoStepCholesky.f90:378-416 ---------------- */
    if (want_rkpq && N > 0) {
        int64_t msd = res->max_subset_dim;
        res->rkpq = (double *)calloc((size_t)N * (msd > 0 ? msd : 1) * res->nsubsets, sizeof(double));
        double *W = (double *)malloc(sizeof(double) * (size_t)(msd > 0 ? msd : 1) * N);
        for (int64_t X = 0; X < res->nsubsets; ++X) {
            memset(W, 0, sizeof(double) * (size_t)msd * N);
            int64_t lo = res->subsetbounds[2 * X], hi = res->subsetbounds[2 * X + 1];
            if (lo < 0) continue;
            /* chol2_Vabrs, Step2.f90:242-363 */
#pragma omp parallel for collapse(2) schedule(dynamic)
            for (int64_t L = 0; L < npsp; ++L)
                for (int64_t sab = lo; sab <= hi; ++sab) {
                    int64_t scd = res->pivshellpairs[L];
                    int A = res->shellpairs[2 * sab], B = res->shellpairs[2 * sab + 1];
                    int C = res->shellpairs[2 * scd], Dd = res->shellpairs[2 * scd + 1];
                    int Na = nfunc(b, A), Nb = nfunc(b, B), Nc = nfunc(b, C), Nd = nfunc(b, Dd);
                    double *Vq = (double *)malloc(sizeof(double) * (size_t)Na * Nb * Nc * Nd);
                    quartet_into(b, A, B, C, Dd, kappa, Vq);
                    int64_t ab0 = res->shellpairloc[3 * sab + 1], rs0 = res->pivshellpairloc[L];
                    for (int rs = 0; rs < res->pivshellpairdim[L]; ++rs) {
                        int64_t cdi = res->pivorbpairs[rs0 + rs];
                        for (int bb = 0; bb < Nb; ++bb)
                            for (int a = 0; a < Na; ++a) {
                                int64_t al = pair_local(a, bb, Na, A == B);
                                if (al < 0) continue;
                                W[(ab0 + al) + (size_t)msd * (rs0 + rs)] =
                                    Vq[a + (size_t)Na * bb + (size_t)Na * Nb * cdi];
                            }
                    }
                    free(Vq);
                }
            /* real_abT: Rkpq(:,:,X) = InvL * W^T */
            g_stats[3] += 2.0 * (double)N * N * msd;
            double *R = res->rkpq + (size_t)N * msd * X;
            const double *Inv = res->inv_l;
#pragma omp parallel for schedule(static)
            for (int64_t pq = 0; pq < msd; ++pq)
                for (int64_t k = 0; k < N; ++k) {
                    double s = 0.0;
                    for (int64_t J = 0; J <= k; ++J) s += Inv[k + N * J] * W[pq + (size_t)msd * J];
                    R[k + (size_t)N * pq] = s;
                }
        }
        free(W);
    }
    return 0;
}

void orc_chol_free(orc_chol *r)
{
    free(r->shellpairs); free(r->shellpairloc); free(r->shellpairdim); free(r->subsetdim);
    free(r->subsetbounds); free(r->pivots); free(r->pivot_order); free(r->pivot_dmax);
    free(r->pivshellpairs); free(r->pivshellpairloc); free(r->pivshellpairdim);
    free(r->pivorbpairs); free(r->inv_l); free(r->rkpq);
    memset(r, 0, sizeof(*r));
}

/* ====================================================================== */
/* AO -> MO, Cholesky_Gammcor.f90:143-332                                  */
/* ====================================================================== */
int orc_mo_transf(const orc_chol *c, const orc_basis *b, const int *shell_loc,
                  const double *CA, int64_t ldca, int64_t a0, int64_t a1,
                  const double *CB, int64_t ldcb, int64_t b0, int64_t b1,
                  int nthreads, double *rkab)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    if (!c->rkpq) return -1;
    int64_t N = c->nvecs, NA = a1 - a0 + 1, NB = b1 - b0 + 1, nao = c->nao, msd = c->max_subset_dim;
    /* Step 1: W(k, a, p) = sum_pq R(k,pq) C(q,a) [+ both triangle halves] */
    double *W = (double *)calloc((size_t)N * NA * nao, sizeof(double));
    for (int64_t X = 0; X < c->nsubsets; ++X) {
        int64_t lo = c->subsetbounds[2 * X], hi = c->subsetbounds[2 * X + 1];
        if (lo < 0) continue;
        const double *R = c->rkpq + (size_t)N * msd * X;
        for (int64_t s = lo; s <= hi; ++s) {
            int A = c->shellpairs[2 * s], B = c->shellpairs[2 * s + 1];
            int Na = nfunc(b, A), Nb = nfunc(b, B);
            int64_t LocA = shell_loc[A], LocB = shell_loc[B];
            int64_t pq = c->shellpairloc[3 * s + 1];
            for (int bb = 0; bb < Nb; ++bb)
                for (int a = (A == B) ? bb : 0; a < Na; ++a, ++pq) {
                    int64_t p = LocA + a, q = LocB + bb;
                    const double *r = R + (size_t)N * pq;
#pragma omp parallel for schedule(static)
                    for (int64_t aa = 0; aa < NA; ++aa) {
                        double cq = CA[q + ldca * (a0 + aa)], cp = CA[p + ldca * (a0 + aa)];
                        double *wp = W + (size_t)N * (aa + NA * p);
                        double *wq = W + (size_t)N * (aa + NA * q);
                        if (p == q) {
                            for (int64_t k = 0; k < N; ++k) wp[k] += r[k] * cq;
                        } else {
                            for (int64_t k = 0; k < N; ++k) { wp[k] += r[k] * cq; wq[k] += r[k] * cp; }
                        }
                    }
                }
        }
    }
    g_stats[4] += 2.0 * (double)N * NA * nao * nao + 2.0 * (double)N * NA * NB * nao;
    /* Step 2: Rab(:, a, b) += sum_p W(:, a, p) CB(p, b) */
#pragma omp parallel for schedule(static)
    for (int64_t bb = 0; bb < NB; ++bb)
        for (int64_t aa = 0; aa < NA; ++aa) {
            double *out = rkab + (size_t)N * (aa + NA * bb);
            for (int64_t k = 0; k < N; ++k) out[k] = 0.0;
            for (int64_t p = 0; p < nao; ++p) {
                double cb = CB[p + ldcb * (b0 + bb)];
                const double *w = W + (size_t)N * (aa + NA * p);
                for (int64_t k = 0; k < N; ++k) out[k] += w[k] * cb;
            }
        }
    free(W);
    return 0;
}

/* ====================================================================== */
/* Dense (pq|rs) and the Coulomb energy gradient (new capability; no       */
/* reference counterpart -- checked by central finite differences).       */
/* ====================================================================== */
int orc_eri_full(const orc_basis *b, const int *shell_loc, int64_t nao, double kappa,
                 int nthreads, double *out)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    if (orc_boys_init(4 * ORC_MAXL) != 0) return -2;
    int nsh = b->nshells;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int A = 0; A < nsh; ++A)
        for (int B = 0; B < nsh; ++B)
            for (int C = 0; C < nsh; ++C)
                for (int Dd = 0; Dd < nsh; ++Dd) {
                    int Na = nfunc(b, A), Nb = nfunc(b, B), Nc = nfunc(b, C), Nd = nfunc(b, Dd);
                    double *V = (double *)malloc(sizeof(double) * (size_t)Na * Nb * Nc * Nd);
                    orc_eri_quartet(b, A, B, C, Dd, kappa, V);
                    for (int d = 0; d < Nd; ++d)
                        for (int c = 0; c < Nc; ++c)
                            for (int bb = 0; bb < Nb; ++bb)
                                for (int a = 0; a < Na; ++a) {
                                    int64_t p = shell_loc[A] + a, q = shell_loc[B] + bb;
                                    int64_t r = shell_loc[C] + c, s = shell_loc[Dd] + d;
                                    out[p + nao * (q + nao * (r + nao * s))] =
                                        V[a + (size_t)Na * (bb + (size_t)Nb * (c + (size_t)Nc * d))];
                                }
                    free(V);
                }
    return 0;
}

/* Derivative of a contracted Cartesian quartet with respect to the centre of
 * shell `which` (0..3): d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x phi_{a-1x},
 * evaluated per primitive (exponent-weighted coefficients for the raised
 * shell).  Output Gd[xyz][a,b,c,d] Cartesian, a fastest. */
static void cart_quartet_deriv(const orc_basis *b, const int sh[4], int which, double kappa, double *Gd)
{
    int l[4], n[4];
    for (int i = 0; i < 4; ++i) { l[i] = b->L[sh[i]]; n[i] = NCART(l[i]); }
    size_t tot = (size_t)n[0] * n[1] * n[2] * n[3];
    const double *R[4]; int np[4]; const double *ex[4], *cf[4];
    for (int i = 0; i < 4; ++i) {
        R[i] = b->coords + 3 * sh[i]; np[i] = b->nprim[sh[i]];
        ex[i] = b->exps + b->prim_off[sh[i]]; cf[i] = b->coefs + b->prim_off[sh[i]];
    }
    double cup[64];
    for (int p = 0; p < np[which]; ++p) cup[p] = 2.0 * ex[which][p] * cf[which][p];
    int lu[4] = {l[0], l[1], l[2], l[3]};
    lu[which] += 1;
    int nu[4] = {n[0], n[1], n[2], n[3]};
    nu[which] = NCART(lu[which]);
    size_t totu = (size_t)nu[0] * nu[1] * nu[2] * nu[3];
    double *Gu = (double *)malloc(sizeof(double) * totu);
    const double *cfu[4] = {cf[0], cf[1], cf[2], cf[3]};
    cfu[which] = cup;
    cart_quartet_any(lu[0], lu[1], lu[2], lu[3], R[0], R[1], R[2], R[3],
                 np[0], ex[0], cfu[0], np[1], ex[1], cfu[1], np[2], ex[2], cfu[2], np[3], ex[3], cfu[3],
                 kappa, Gu);
    double *Gl = NULL;
    int nl[4] = {n[0], n[1], n[2], n[3]};
    if (l[which] > 0) {
        int ll[4] = {l[0], l[1], l[2], l[3]};
        ll[which] -= 1;
        nl[which] = NCART(ll[which]);
        Gl = (double *)malloc(sizeof(double) * (size_t)nl[0] * nl[1] * nl[2] * nl[3]);
        cart_quartet_any(ll[0], ll[1], ll[2], ll[3], R[0], R[1], R[2], R[3],
                     np[0], ex[0], cf[0], np[1], ex[1], cf[1], np[2], ex[2], cf[2], np[3], ex[3], cf[3],
                     kappa, Gl);
    }
    int strides[4] = {1, n[0], n[0] * n[1], n[0] * n[1] * n[2]};
    int su[4] = {1, nu[0], nu[0] * nu[1], nu[0] * nu[1] * nu[2]};
    int sl[4] = {1, nl[0], nl[0] * nl[1], nl[0] * nl[1] * nl[2]};
    int base = CART_OFF(l[which]), baseu = CART_OFF(l[which] + 1), basel = l[which] > 0 ? CART_OFF(l[which] - 1) : 0;
    for (size_t idx = 0; idx < tot; ++idx) {
        int ii[4];
        size_t r = idx;
        for (int i = 0; i < 4; ++i) { ii[i] = (int)(r % n[i]); r /= n[i]; }
        int g = base + ii[which];
        int cx = g_cx[g], cy = g_cy[g], cz = g_cz[g];
        for (int ax = 0; ax < 3; ++ax) {
            int ux = cx + (ax == 0), uy = cy + (ax == 1), uz = cz + (ax == 2);
            int upos = cart_pos(uy, uz);
            size_t iu = 0;
            for (int i = 0; i < 4; ++i) iu += (size_t)((i == which) ? upos : ii[i]) * su[i];
            double v = Gu[iu];
            int comp = (ax == 0) ? cx : ((ax == 1) ? cy : cz);
            if (comp > 0) {
                int dx = cx - (ax == 0), dy = cy - (ax == 1), dz = cz - (ax == 2);
                int dpos = cart_pos(dy, dz);
                size_t il = 0;
                for (int i = 0; i < 4; ++i) il += (size_t)((i == which) ? dpos : ii[i]) * sl[i];
                v -= comp * Gl[il];
            }
            Gd[(size_t)ax * tot + idx] = v;
        }
        (void)baseu; (void)basel; (void)strides;
    }
    free(Gu); free(Gl);
}

int orc_coulomb_energy_grad(const orc_basis *b, const int *shell_atom, int natoms,
                            const int *shell_loc, const double *Dm, int64_t nao,
                            double kappa, int nthreads, double *energy, double *grad)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    if (orc_boys_init(4 * ORC_MAXL) != 0) return -2;
    int nsh = b->nshells;
    double e = 0.0;
    for (int i = 0; i < 3 * natoms; ++i) grad[i] = 0.0;
#pragma omp parallel
    {
        double *gloc = (double *)calloc(3 * natoms, sizeof(double));
        double eloc = 0.0;
#pragma omp for collapse(2) schedule(dynamic)
        for (int A = 0; A < nsh; ++A)
            for (int B = 0; B < nsh; ++B)
                for (int C = 0; C < nsh; ++C)
                    for (int Dd = 0; Dd < nsh; ++Dd) {
                        int sh[4] = {A, B, C, Dd};
                        int n[4], nf[4]; const double *T[4];
                        for (int i = 0; i < 4; ++i) {
                            n[i] = NCART(b->L[sh[i]]); nf[i] = nfunc(b, sh[i]);
                            T[i] = b->T + b->T_off[sh[i]];
                        }
                        size_t tot = (size_t)n[0] * n[1] * n[2] * n[3];
                        size_t totf = (size_t)nf[0] * nf[1] * nf[2] * nf[3];
                        /* density block Dab Dcd in the function basis */
                        double *V = (double *)malloc(sizeof(double) * totf);
                        orc_eri_quartet(b, A, B, C, Dd, kappa, V);
                        double *Gd = (double *)malloc(sizeof(double) * 3 * tot);
                        double *Vt = (double *)malloc(sizeof(double) * totf);
                        for (size_t idx = 0; idx < totf; ++idx) {
                            size_t r = idx; int ii[4];
                            for (int i = 0; i < 4; ++i) { ii[i] = (int)(r % nf[i]); r /= nf[i]; }
                            double w = Dm[(shell_loc[A] + ii[0]) + nao * (shell_loc[B] + ii[1])] *
                                       Dm[(shell_loc[C] + ii[2]) + nao * (shell_loc[Dd] + ii[3])];
                            eloc += 0.5 * w * V[idx];
                        }
                        for (int which = 0; which < 3; ++which) {
                            cart_quartet_deriv(b, sh, which, kappa, Gd);
                            for (int ax = 0; ax < 3; ++ax) {
                                transform4(Gd + (size_t)ax * tot, n, T, nf, Vt);
                                double s = 0.0;
                                for (size_t idx = 0; idx < totf; ++idx) {
                                    size_t r = idx; int ii[4];
                                    for (int i = 0; i < 4; ++i) { ii[i] = (int)(r % nf[i]); r /= nf[i]; }
                                    s += Dm[(shell_loc[A] + ii[0]) + nao * (shell_loc[B] + ii[1])] *
                                         Dm[(shell_loc[C] + ii[2]) + nao * (shell_loc[Dd] + ii[3])] * Vt[idx];
                                }
                                s *= 0.5;
                                gloc[3 * shell_atom[sh[which]] + ax] += s;
                                gloc[3 * shell_atom[Dd] + ax] -= s;   /* translational invariance */
                            }
                        }
                        free(V); free(Gd); free(Vt);
                    }
#pragma omp critical
        {
            e += eloc;
            for (int i = 0; i < 3 * natoms; ++i) grad[i] += gloc[i];
        }
        free(gloc);
    }
    *energy = e;
    return 0;
}

/* Timing sample of the reference algorithm (test and benchmark
 * infrastructure): n shell quartets (A, B, C, D per quartet, 0-based)
 * evaluated by orc_eri_quartet over `nthreads` OpenMP threads; the integrals
 * are folded into a checksum so that the work is not discarded. */
double orc_eri_quartets_batch(const orc_basis *b, int64_t n, const int *quads, double kappa, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    if (orc_boys_init(4 * ORC_MAXL) != 0) return 0.0;
    double sum = 0.0;
#pragma omp parallel reduction(+ : sum)
    {
        double *V = (double *)malloc(sizeof(double) * 10000);
#pragma omp for schedule(dynamic)
        for (int64_t q = 0; q < n; ++q) {
            const int *s = quads + 4 * q;
            if (orc_eri_quartet(b, s[0], s[1], s[2], s[3], kappa, V) == 0) {
                const int tot = nfunc(b, s[0]) * nfunc(b, s[1]) * nfunc(b, s[2]) * nfunc(b, s[3]);
                for (int i = 0; i < tot; ++i) sum += V[i];
            }
        }
        free(V);
    }
    return sum;
}

/* Exported forms of the Hermite recursions for the fixture tests: R_tuv for
 * t+u+v <= n in level-major order (herm_idx), and the
 * single-centre E^{e}_t, [emax+1][emax+1]. */
void orc_rtuv(int n, const double *F, double alpha, double X, double Y, double Z, double *R)
{
    rtuv(n, F, alpha, X, Y, Z, R);
}

void orc_et_coeffs(int emax, double p, double X, double *E)
{
    et_coeffs(emax, p, X, E);
}
