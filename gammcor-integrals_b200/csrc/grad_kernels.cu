// grad_kernels.cu -- density-contracted Hermite vectors, the dot products that
// give the Coulomb energy and its nuclear gradient, the Coulomb matrix, and
// the dispatch table of the potential kernels (grad_engine.cuh,
// instantiated in grad_pot_*.cu).
#include "grad_engine.cuh"
#include "gci_runtime.h"
#include <mutex>

namespace gci {

// E^{ij}_t of one axis for i <= la + 1, j <= lb + 1 (t <= i + j; zero beyond):
// the two-centre McMurchie-Davidson recursion in P-A and P-B with
// E^{00}_0 = 1 (the Gaussian product factor is applied separately).
struct GradE {
    static constexpr int NI = kMaxL + 2, NT = 2 * kMaxL + 3;
    double e[NI][NI][NT];
};

__device__ static void grad_etab(GradE& E, int la, int lb, double PA, double PB, double h)
{
    for (int i = 0; i < GradE::NI; ++i)
        for (int j = 0; j < GradE::NI; ++j)
            for (int t = 0; t < GradE::NT; ++t) E.e[i][j][t] = 0.0;
    E.e[0][0][0] = 1.0;
    for (int i = 0; i <= la; ++i)
        for (int t = 0; t <= i + 1; ++t) {
            double v = PA * E.e[i][0][t];
            if (t >= 1) v += h * E.e[i][0][t - 1];
            if (t + 1 <= i) v += (double)(t + 1) * E.e[i][0][t + 1];
            E.e[i + 1][0][t] = v;
        }
    for (int j = 0; j <= lb; ++j)
        for (int i = 0; i <= la + 1; ++i)
            for (int t = 0; t <= i + j + 1; ++t) {
                double v = PB * E.e[i][j][t];
                if (t >= 1) v += h * E.e[i][j][t - 1];
                if (t + 1 <= i + j) v += (double)(t + 1) * E.e[i][j][t + 1];
                E.e[i][j + 1][t] = v;
            }
}

// One block per shell pair: the Cartesian density block Ds (symmetrised,
// times w_AB, with the norms and spherical transforms of both shells) in
// shared memory, then one thread per kept primitive pair writes its seven
// Hermite vectors (h, gA, gB; grad_hb(L) entries each), its geometry and,
// transposed and signed, its ket vector.
__global__ void k_grad_pair_vectors(const ShellPairDev* __restrict__ pairs, int npairs,
                                    const int64_t* __restrict__ gbase, const int* __restrict__ level_beg,
                                    const int* __restrict__ level_n, const int64_t* __restrict__ vec_off,
                                    const int64_t* __restrict__ hk_off, const double* __restrict__ xyz,
                                    const int* __restrict__ poff, const double* __restrict__ exps,
                                    const double* __restrict__ coefs, const int* __restrict__ plist,
                                    const double* __restrict__ tmat, const int* __restrict__ toff,
                                    const int* __restrict__ nfunc, const int* __restrict__ loc,
                                    const double* __restrict__ D, int64_t ldd, double* __restrict__ mP,
                                    double* __restrict__ mX, double* __restrict__ mY, double* __restrict__ mZ,
                                    double* __restrict__ vecs, double* __restrict__ hk, int* __restrict__ ppair)
{
    __shared__ double Dc[ncart(kMaxL) * ncart(kMaxL)];
    for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
        const ShellPairDev sp = pairs[p];
        const int s1 = sp.s1, s2 = sp.s2, la = sp.l1, lb = sp.l2, L = la + lb;
        const int nc1 = ncart(la), nc2 = ncart(lb), nf1 = nfunc[s1], nf2 = nfunc[s2];
        const double* T1 = tmat + toff[s1];
        const double* T2 = tmat + toff[s2];
        const int64_t l1 = loc[s1], l2 = loc[s2];
        const double w = (s1 != s2) ? 2.0 : 1.0;
        __syncthreads();
        for (int e = threadIdx.x; e < nc1 * nc2; e += blockDim.x) {
            const int a = e / nc2, b = e - a * nc2;
            double acc = 0.0;
            for (int mb = 0; mb < nf2; ++mb) {
                double row = 0.0;
                for (int ma = 0; ma < nf1; ++ma) {
                    const int64_t pp = l1 + ma, qq = l2 + mb;
                    row += T1[ma * nc1 + a] * 0.5 * (D[pp + ldd * qq] + D[qq + ldd * pp]);
                }
                acc += row * T2[mb * nc2 + b];
            }
            Dc[e] = w * acc;
        }
        __syncthreads();
        const double ax = xyz[3 * s1], ay = xyz[3 * s1 + 1], az = xyz[3 * s1 + 2];
        const double bx = xyz[3 * s2], by = xyz[3 * s2 + 1], bz = xyz[3 * s2 + 2];
        const double r2 = (ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz);
        const int HB = grad_hb(L);
        const int HL = herm_n(L);
        for (int i = threadIdx.x; i < sp.npp; i += blockDim.x) {
            const int code = plist[sp.list_off + i];
            const int ga = code & 0xff, gb = code >> 8;
            const double ea = exps[poff[s1] + ga], eb = exps[poff[s2] + gb];
            const double ca = coefs[poff[s1] + ga], cb = coefs[poff[s2] + gb];
            const double P = ea + eb;
            const double px = (ea * ax + eb * bx) / P, py = (ea * ay + eb * by) / P, pz = (ea * az + eb * bz) / P;
            const double K = exp(-ea * eb / P * r2) * ca * cb;
            const double h = 1.0 / (2.0 * P);
            GradE Ex, Ey, Ez;
            grad_etab(Ex, la, lb, px - ax, px - bx, h);
            grad_etab(Ey, la, lb, py - ay, py - by, h);
            grad_etab(Ez, la, lb, pz - az, pz - bz, h);
            const int64_t g = gbase[p] + i;
            const int64_t li = g - level_beg[L];
            double* vg = vecs + vec_off[L] + li * (int64_t)(kGradVec * HB);
            for (int c = 0; c < kGradVec * HB; ++c) vg[c] = 0.0;
            for (int a = 0; a < nc1; ++a) {
                const int A = cart_off(la) + a;
                const int axx = cart_x(A), ayy = cart_y(A), azz = cart_z(A);
                for (int b = 0; b < nc2; ++b) {
                    const double d = K * Dc[a * nc2 + b];
                    if (d == 0.0) continue;
                    const int B = cart_off(lb) + b;
                    const int bxx = cart_x(B), byy = cart_y(B), bzz = cart_z(B);
                    // (t, u, v) up to one unit above the pair's range on each axis, but
                    // only up to level L + 1 in total: every nonzero product lies there,
                    // and the vector block of this primitive pair ends there
                    for (int v = 0; v <= azz + bzz + 1; ++v) {
                        const double z0 = Ez.e[azz][bzz][v];
                        const double zA = 2.0 * ea * Ez.e[azz + 1][bzz][v] - (azz > 0 ? azz * Ez.e[azz - 1][bzz][v] : 0.0);
                        const double zB = 2.0 * eb * Ez.e[azz][bzz + 1][v] - (bzz > 0 ? bzz * Ez.e[azz][bzz - 1][v] : 0.0);
                        for (int u = 0; u <= ayy + byy + 1 && u + v <= L + 1; ++u) {
                            const double y0 = Ey.e[ayy][byy][u];
                            const double yA = 2.0 * ea * Ey.e[ayy + 1][byy][u] - (ayy > 0 ? ayy * Ey.e[ayy - 1][byy][u] : 0.0);
                            const double yB = 2.0 * eb * Ey.e[ayy][byy + 1][u] - (byy > 0 ? byy * Ey.e[ayy][byy - 1][u] : 0.0);
                            for (int t = 0; t <= axx + bxx + 1 && t + u + v <= L + 1; ++t) {
                                const double x0 = Ex.e[axx][bxx][t];
                                const double xA = 2.0 * ea * Ex.e[axx + 1][bxx][t] - (axx > 0 ? axx * Ex.e[axx - 1][bxx][t] : 0.0);
                                const double xB = 2.0 * eb * Ex.e[axx][bxx + 1][t] - (bxx > 0 ? bxx * Ex.e[axx][bxx - 1][t] : 0.0);
                                const int hh = herm_idx(t, u, v);
                                vg[0 * HB + hh] += d * x0 * y0 * z0;
                                vg[1 * HB + hh] += d * xA * y0 * z0;
                                vg[2 * HB + hh] += d * x0 * yA * z0;
                                vg[3 * HB + hh] += d * x0 * y0 * zA;
                                vg[4 * HB + hh] += d * xB * y0 * z0;
                                vg[5 * HB + hh] += d * x0 * yB * z0;
                                vg[6 * HB + hh] += d * x0 * y0 * zB;
                            }
                        }
                    }
                }
            }
            mP[g] = P; mX[g] = px; mY[g] = py; mZ[g] = pz;
            ppair[g] = p;
            // ket role: (-1)^{tau+nu+phi} h(tau), transposed within the level
            const int64_t nL = level_n[L];
            for (int tau = 0; tau < HL; ++tau) {
                const int s = herm_level(tau);
                hk[hk_off[L] + (int64_t)tau * nL + li] = (s & 1) ? -vg[tau] : vg[tau];
            }
        }
    }
}

// One thread per primitive pair: the seven dot products of its vectors with
// its potential, out[g * 7 + c] (c = 0: h.V, 1..3: gA.V, 4..6: gB.V).
__global__ void k_grad_dots(int64_t beg, int64_t n, int HB, const double* __restrict__ vecs,
                            const double* __restrict__ V, double* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double* vg = vecs + i * (int64_t)(kGradVec * HB);
        const double* vi = V + i * (int64_t)HB;
        for (int c = 0; c < kGradVec; ++c) {
            double s = 0.0;
            for (int h = 0; h < HB; ++h) s += vg[c * HB + h] * vi[h];
            out[(beg + i) * kGradVec + c] = s;
        }
    }
}

// Coulomb matrix J_pq = sum_rs (pq|rs) Ds_rs: one block per shell pair; a
// thread per Cartesian pair (a, b) contracts the pair's primitive-pair
// records (K c_a c_b and the Hermite products E^{ab}_tuv, as the ERI kernels
// read them) with the potentials, then the block applies the two shells'
// transforms and writes the (s1, s2) block and its transpose.
__global__ void k_grad_coulomb_matrix(const ShellPairDev* __restrict__ pairs, int npairs,
                                      const int64_t* __restrict__ gbase, const int* __restrict__ level_beg,
                                      const int64_t* __restrict__ pot_off, const double* __restrict__ V,
                                      const double* __restrict__ pp, const double* __restrict__ tmat,
                                      const int* __restrict__ toff, const int* __restrict__ nfunc,
                                      const int* __restrict__ loc, double* __restrict__ J, int64_t ldj)
{
    __shared__ double Jc[ncart(kMaxL) * ncart(kMaxL)];
    __shared__ double Jh[(2 * kMaxL + 1) * ncart(kMaxL)];
    for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
        const ShellPairDev sp = pairs[p];
        const int s1 = sp.s1, s2 = sp.s2, la = sp.l1, lb = sp.l2, L = la + lb;
        const int nc1 = ncart(la), nc2 = ncart(lb), nf1 = nfunc[s1], nf2 = nfunc[s2];
        const int HB = grad_hb(L);
        const int rs = pp_record(la, lb), po = pp_prod_off(la, lb);
        __syncthreads();
        for (int e = threadIdx.x; e < nc1 * nc2; e += blockDim.x) {
            int off = 0;
            for (int f = 0; f < e; ++f) off += pair_supp(la, lb, f);
            const int ex = pair_x(la, lb, e), ey = pair_y(la, lb, e), ez = pair_z(la, lb, e);
            double acc = 0.0;
            for (int i = 0; i < sp.npp; ++i) {
                const double* rec = pp + sp.rec_off + (int64_t)i * rs;
                const double* prod = rec + po + off;
                const int64_t g = gbase[p] + i;
                const double* vi = V + pot_off[L] + (g - level_beg[L]) * (int64_t)HB;
                double s = 0.0;
                int c = 0;
                for (int v = 0; v <= ez; ++v)
                    for (int u = 0; u <= ey; ++u)
                        for (int t = 0; t <= ex; ++t) s += prod[c++] * vi[herm_idx(t, u, v)];
                acc += rec[4] * s;
            }
            Jc[e] = acc;
        }
        __syncthreads();
        const double* T1 = tmat + __ldg(toff + s1);
        const double* T2 = tmat + __ldg(toff + s2);
        for (int e = threadIdx.x; e < nf1 * nc2; e += blockDim.x) {
            const int ma = e / nc2, b = e - ma * nc2;
            double acc = 0.0;
            for (int a = 0; a < nc1; ++a) acc += T1[ma * nc1 + a] * Jc[a * nc2 + b];
            Jh[e] = acc;
        }
        __syncthreads();
        const int64_t l1 = loc[s1], l2 = loc[s2];
        for (int e = threadIdx.x; e < nf1 * nf2; e += blockDim.x) {
            const int ma = e / nf2, mb = e - ma * nf2;
            double acc = 0.0;
            for (int b = 0; b < nc2; ++b) acc += Jh[ma * nc2 + b] * T2[mb * nc2 + b];
            J[(l1 + ma) + ldj * (l2 + mb)] = acc;
            J[(l2 + mb) + ldj * (l1 + ma)] = acc;
        }
    }
}

static GradLaunchFn g_grad_launch[kGradMaxL + 1][kGradMaxL + 1];

cudaError_t grad_module_init()
{
    // the table is filled once; concurrent first calls wait for it
    static std::once_flag once;
    std::call_once(once, [] {
        register_grad_pot_a(g_grad_launch);
        register_grad_pot_b(g_grad_launch);
        register_grad_pot_c(g_grad_launch);
    });
    return cudaSuccess;
}

cudaError_t grad_pair_vectors_launch(const ShellPairDev* pairs, int npairs, const int64_t* gbase,
                                     const int* level_beg, const int* level_n, const int64_t* vec_off,
                                     const int64_t* hk_off, const double* xyz, const int* poff, const double* exps,
                                     const double* coefs, const int* plist, const double* tmat, const int* toff,
                                     const int* nfunc, const int* loc, const double* D, int64_t ldd, double* mP,
                                     double* mX, double* mY, double* mZ, double* vecs, double* hk, int* ppair,
                                     cudaStream_t st)
{
    if (npairs <= 0) return cudaSuccess;
    const int blocks = npairs < 148 * 32 ? npairs : 148 * 32;
    k_grad_pair_vectors<<<blocks, 64, 0, st>>>(pairs, npairs, gbase, level_beg, level_n, vec_off, hk_off, xyz, poff,
                                               exps, coefs, plist, tmat, toff, nfunc, loc, D, ldd, mP, mX, mY, mZ,
                                               vecs, hk, ppair);
    count_launch();
    return cudaGetLastError();
}

cudaError_t grad_potential_launch(int L1, int L2, const GradPotArgs& a, cudaStream_t st)
{
    if (L1 < 0 || L2 < 0 || L1 > kGradMaxL || L2 > kGradMaxL || !g_grad_launch[L1][L2]) return cudaErrorInvalidValue;
    if (a.nbra <= 0 || a.nket <= 0) return cudaSuccess;
    g_grad_launch[L1][L2](a, st);
    count_launch();
    return cudaGetLastError();
}

cudaError_t grad_dots_launch(int64_t beg, int64_t n, int HB, const double* vecs, const double* V, double* out,
                             cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    int64_t blocks = (n + 127) / 128;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_grad_dots<<<(unsigned)blocks, 128, 0, st>>>(beg, n, HB, vecs, V, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t grad_coulomb_matrix_launch(const ShellPairDev* pairs, int npairs, const int64_t* gbase,
                                       const int* level_beg, const int64_t* pot_off, const double* V, const double* pp,
                                       const double* tmat, const int* toff, const int* nfunc, const int* loc,
                                       double* J, int64_t ldj, cudaStream_t st)
{
    if (npairs <= 0) return cudaSuccess;
    const int blocks = npairs < 148 * 32 ? npairs : 148 * 32;
    k_grad_coulomb_matrix<<<blocks, 128, 0, st>>>(pairs, npairs, gbase, level_beg, pot_off, V, pp, tmat, toff, nfunc,
                                                  loc, J, ldj);
    count_launch();
    return cudaGetLastError();
}

} // namespace gci
