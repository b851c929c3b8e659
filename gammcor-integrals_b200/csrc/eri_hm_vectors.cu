// eri_hm_vectors.cu -- the pair Hermite vectors of the Hermite-matrix ERI
// kernels (eri_hermite.cuh) and the launch table of those kernels.
//
// A vector element is the Hermite coefficient of one (spherical, normalised)
// function pair of a primitive pair,
//     K c c sum_{a in A, b in B} T_A(f_a, a) T_B(f_b, b) Ex^{ab}_t Ey^{ab}_u Ez^{ab}_v,
// the normalisation and solid-harmonic transforms of the reference
// (auto2e_SpherTransf.f90, auto2e_Normalize_*, sphergto.f90:184-211)
// applied to the two-centre Hermite coefficients of the primitive-pair
// record (k_pair_records).  Elements are written directly in the fragment
// order the DMMA products read.
#include "eri_hermite.cuh"
#include "gci_runtime.h"
#include <mutex>

namespace gci {

// Coefficient of Hermite index (t,u,v) of the function pair (f1, f2) of the
// canonical shells (s1, s2) of a pair in primitive-pair record `rec`.
__device__ static double hm_element(const ShellPairDev& d, const double* __restrict__ rec, int f1, int f2, int t,
                                    int u, int v, const double* __restrict__ tmat, const int* __restrict__ toff)
{
    const int la = d.l1, lb = d.l2;
    const int n1 = ncart(la), n2 = ncart(lb);
    const int ne = e2_size(la, lb);
    const double* __restrict__ Ex = rec + 8;
    const double* __restrict__ Ey = Ex + ne;
    const double* __restrict__ Ez = Ey + ne;
    const double* __restrict__ T1 = tmat + __ldg(toff + d.s1) + f1 * n1;
    const double* __restrict__ T2 = tmat + __ldg(toff + d.s2) + f2 * n2;
    double sum = 0.0;
    for (int c1 = 0; c1 < n1; ++c1) {
        const double w1 = __ldg(T1 + c1);
        if (w1 == 0.0) continue;
        const int g1 = cart_off(la) + c1;
        const int x1 = cart_x(g1), y1 = cart_y(g1), z1 = cart_z(g1);
        for (int c2 = 0; c2 < n2; ++c2) {
            const double w2 = __ldg(T2 + c2);
            if (w2 == 0.0) continue;
            const int g2 = cart_off(lb) + c2;
            const int x2 = cart_x(g2), y2 = cart_y(g2), z2 = cart_z(g2);
            if (t > x1 + x2 || u > y1 + y2 || v > z1 + z2) continue;
            sum += w1 * w2 * Ex[e2_off(la, x1, x2) + t] * Ey[e2_off(la, y1, y2) + u] * Ez[e2_off(la, z1, z2) + v];
        }
    }
    return sum * rec[4];
}

// Stored-orientation function code f = f_first + N_first f_second -> canonical (f1, f2).
__device__ __forceinline__ void hm_canon(const ShellPairDev& d, const int* __restrict__ nfunc, int f, int& f1, int& f2)
{
    const int first = d.swap ? d.s2 : d.s1;
    const int nfirst = __ldg(nfunc + first);
    const int fa = f % nfirst, fb = f / nfirst;
    f1 = d.swap ? fb : fa;
    f2 = d.swap ? fa : fb;
}

// Row vectors of the listed pairs: per primitive pair [MTO][2 MT][32], element
// (m, ks, l) = Er(r = 8 m + l/4, h = 4 ks + l%4); one block per pair.
__global__ void k_hm_rowvec(const int* __restrict__ ids, int nids, const ShellPairDev* __restrict__ pairs,
                            const double* __restrict__ pp, const int64_t* __restrict__ off,
                            const double* __restrict__ tmat, const int* __restrict__ toff,
                            const int* __restrict__ nfunc, double* __restrict__ vec)
{
    for (int q = blockIdx.x; q < nids; q += gridDim.x) {
        const int id = ids[q];
        const ShellPairDev d = pairs[id];
        const int L = d.l1 + d.l2;
        const int H = herm_n(L), MT2 = 2 * hm_mt(L), stride = hm_row_stride(L);
        const int nR = __ldg(nfunc + d.s1) * __ldg(nfunc + d.s2);
        const int rs = pp_record(d.l1, d.l2);
        double* __restrict__ out = vec + off[id];
        const int64_t n = (int64_t)d.npp * stride;
        for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
            const int i = (int)(e / stride);
            const int w = (int)(e - (int64_t)i * stride);
            const int l = w & 31, f = w >> 5;
            const int m = f / MT2, ks = f - m * MT2;
            const int r = 8 * m + (l >> 2), h = 4 * ks + (l & 3);
            double val = 0.0;
            if (r < nR && h < H) {
                int f1, f2;
                hm_canon(d, nfunc, r, f1, f2);
                val = hm_element(d, pp + d.rec_off + (size_t)i * rs, f1, f2, herm_t(h), herm_u(h), herm_v(h), tmat,
                                 toff);
            }
            out[e] = val;
        }
    }
}

// Column vectors of the chunks: per primitive pair [KT][NT][32], element
// (ks, n, l) = (-1)^|g| Ec(g = 4 ks + l%4, J = 8 n + l/4); one block per chunk.
__global__ void k_hm_colvec(const HmChunk* __restrict__ chunks, int nchunks, const ShellPairDev* __restrict__ pairs,
                            const double* __restrict__ pp, const int* __restrict__ colfun,
                            const double* __restrict__ tmat, const int* __restrict__ toff,
                            const int* __restrict__ nfunc, double* __restrict__ vec)
{
    for (int q = blockIdx.x; q < nchunks; q += gridDim.x) {
        const HmChunk ch = chunks[q];
        const ShellPairDev d = pairs[ch.pair];
        const int L = d.l1 + d.l2;
        const int H = herm_n(L), stride = hm_col_stride(L, ch.nt);
        const int rs = pp_record(d.l1, d.l2);
        double* __restrict__ out = vec + ch.vec_off;
        const int64_t n = (int64_t)d.npp * stride;
        for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
            const int k = (int)(e / stride);
            const int w = (int)(e - (int64_t)k * stride);
            const int l = w & 31, f = w >> 5;
            const int ks = f / ch.nt, nn = f - ks * ch.nt;
            const int g = 4 * ks + (l & 3), J = 8 * nn + (l >> 2);
            double val = 0.0;
            if (g < H && J < ch.ncol) {
                int f1, f2;
                hm_canon(d, nfunc, colfun[ch.col_off + J], f1, f2);
                const int t = herm_t(g), u = herm_u(g), v = herm_v(g);
                val = hm_element(d, pp + d.rec_off + (size_t)k * rs, f1, f2, t, u, v, tmat, toff);
                if ((t + u + v) & 1) val = -val;
            }
            out[e] = val;
        }
    }
}

cudaError_t hm_rowvec_launch(const int* ids, int nids, const ShellPairDev* pairs, const double* pp,
                             const int64_t* off, const double* tmat, const int* toff, const int* nfunc, double* vec,
                             cudaStream_t st)
{
    if (nids <= 0) return cudaSuccess;
    const int blocks = nids < 148 * 32 ? nids : 148 * 32;
    k_hm_rowvec<<<blocks, 256, 0, st>>>(ids, nids, pairs, pp, off, tmat, toff, nfunc, vec);
    count_launch();
    return cudaGetLastError();
}

cudaError_t hm_colvec_launch(const HmChunk* chunks, int nchunks, const ShellPairDev* pairs, const double* pp,
                             const int* colfun, const double* tmat, const int* toff, const int* nfunc, double* vec,
                             cudaStream_t st)
{
    if (nchunks <= 0) return cudaSuccess;
    const int blocks = nchunks < 148 * 32 ? nchunks : 148 * 32;
    k_hm_colvec<<<blocks, 256, 0, st>>>(chunks, nchunks, pairs, pp, colfun, tmat, toff, nfunc, vec);
    count_launch();
    return cudaGetLastError();
}

static HmLaunchFn g_hm[kMaxPairL + 1][kMaxPairL + 1][kHmMaxNT];

static void hm_register()
{
    register_hm_0(g_hm);
    register_hm_1(g_hm);
    register_hm_2(g_hm);
    register_hm_3(g_hm);
    register_hm_4(g_hm);
    register_hm_5(g_hm);
    register_hm_6(g_hm);
}

cudaError_t hm_launch(int L1, int L2, int nt, const HmArgs& a, cudaStream_t st)
{
    static std::once_flag once;
    std::call_once(once, hm_register);
    if (L1 < 0 || L2 < 0 || L1 > kMaxPairL || L2 > kMaxPairL || nt < 1 || nt > hm_max_nt(L1) || !g_hm[L1][L2][nt - 1])
        return cudaErrorInvalidValue;
    cudaError_t e = g_hm[L1][L2][nt - 1](a, st);
    count_launch();
    return e;
}

} // namespace gci
