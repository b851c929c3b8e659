// eri_kernels.cu -- instantiation and dispatch of the class-templated ERI
// kernels, the primitive-pair record kernel and the Boys self-test kernel.
#include "eri_classes.cuh"
#include "gci_runtime.h"
#include <atomic>
#include <mutex>

namespace gci {

// ---------------------------------------------------------------------------
// Primitive-pair records (one block per shell pair, threads over primitive
// pairs, a fastest as in the reference's Ga-inner loop).  The Hermite
// coefficients are the two-centre E^{ij}_t of (x-A)^i (x-B)^j about P
// (McMurchie-Davidson recursion in P-A and P-B), so the ERI kernels need no
// horizontal recurrence: that recurrence, applied after the primitive
// contraction, cancels catastrophically for contracted shells that mix tight
// and diffuse primitives on distant centres.
// ---------------------------------------------------------------------------
__global__ void k_pair_records(const ShellPairDev* __restrict__ pairs, int npairs,
                               const double* __restrict__ xyz, const int* __restrict__ poff,
                               const double* __restrict__ exps, const double* __restrict__ coefs,
                               const int* __restrict__ plist, double* __restrict__ pp)
{
    for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
        const ShellPairDev sp = pairs[p];
        const int la = sp.l1, lb = sp.l2;
        const int rs = pp_record(la, lb);
        const int ne = e2_size(la, lb);
        const int n = sp.npp;
        const double ax = xyz[3 * sp.s1], ay = xyz[3 * sp.s1 + 1], az = xyz[3 * sp.s1 + 2];
        const double bx = xyz[3 * sp.s2], by = xyz[3 * sp.s2 + 1], bz = xyz[3 * sp.s2 + 2];
        const double r2 = (ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int code = plist[sp.list_off + i];
            const int ga = code & 0xff, gb = code >> 8;
            const double ea = exps[poff[sp.s1] + ga], eb = exps[poff[sp.s2] + gb];
            const double ca = coefs[poff[sp.s1] + ga], cb = coefs[poff[sp.s2] + gb];
            const double P = ea + eb;
            const double px = (ea * ax + eb * bx) / P, py = (ea * ay + eb * by) / P, pz = (ea * az + eb * bz) / P;
            double* rec = pp + sp.rec_off + (size_t)i * rs;
            rec[0] = P; rec[1] = px; rec[2] = py; rec[3] = pz;
            rec[4] = exp(-ea * eb / P * r2) * ca * cb;
            rec[5] = px - ax; rec[6] = py - ay; rec[7] = pz - az;
            const double h = 1.0 / (2.0 * P);
            const double PA[3] = {px - ax, py - ay, pz - az};
            const double PB[3] = {px - bx, py - by, pz - bz};
            for (int axis = 0; axis < 3; ++axis) {
                double* E = rec + 8 + axis * ne;
                E[0] = 1.0;
                // raise i on A: E^{i+1,0}
                for (int a = 0; a < la; ++a) {
                    const double* Ei = E + e2_off(la, a, 0);
                    double* En = E + e2_off(la, a + 1, 0);
                    for (int t = 0; t <= a + 1; ++t) {
                        double v = 0.0;
                        if (t >= 1) v += h * Ei[t - 1];
                        if (t <= a) v += PA[axis] * Ei[t];
                        if (t + 1 <= a) v += (double)(t + 1) * Ei[t + 1];
                        En[t] = v;
                    }
                }
                // raise j on B: E^{i,j+1}
                for (int b = 0; b < lb; ++b)
                    for (int a = 0; a <= la; ++a) {
                        const double* Ej = E + e2_off(la, a, b);
                        double* En = E + e2_off(la, a, b + 1);
                        const int m = a + b;
                        for (int t = 0; t <= m + 1; ++t) {
                            double v = 0.0;
                            if (t >= 1) v += h * Ej[t - 1];
                            if (t <= m) v += PB[axis] * Ej[t];
                            if (t + 1 <= m) v += (double)(t + 1) * Ej[t + 1];
                            En[t] = v;
                        }
                    }
            }
            // Hermite products of every Cartesian pair (b fastest), v outer, t inner
            const double* Ex = rec + 8;
            const double* Ey = Ex + ne;
            const double* Ez = Ey + ne;
            double* prod = rec + pp_prod_off(la, lb);
            int c = 0;
            for (int e = 0; e < ncart(la) * ncart(lb); ++e) {
                const int ex = pair_x(la, lb, e), ey = pair_y(la, lb, e), ez = pair_z(la, lb, e);
                const int ox = pair_ox(la, lb, e), oy = pair_oy(la, lb, e), oz = pair_oz(la, lb, e);
                for (int v = 0; v <= ez; ++v)
                    for (int u = 0; u <= ey; ++u) {
                        const double yz = Ey[oy + u] * Ez[oz + v];
                        for (int t = 0; t <= ex; ++t) prod[c++] = Ex[ox + t] * yz;
                    }
            }
        }
    }
}

__global__ void k_boys_eval(int m, int64_t n, const double* __restrict__ x, const double* __restrict__ table,
                            double* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double F[kBoysMaxM + 1];
        boys_fm_rt(m, x[i], table, F);
        for (int k = 0; k <= m; ++k) out[i * (m + 1) + k] = F[k];
    }
}

static LaunchFn g_launch[kNumPairTypes][kNumPairTypes];                   // team kernels (bra types up to (d,d))
static LaunchFn g_launch_kf[kNumKfWidths][kNumPairTypes][kNumPairTypes];  // ket-first kernels where built
// 0 team, 1 + w ket-first of width kf_width(w); read by launches and written by the
// tuner or gci_eri_variant from any thread
static std::atomic<int> g_variant[kNumPairTypes][kNumPairTypes];

static LaunchFn variant_fn(int tb, int tk, int v)
{
    if (v == 0) return g_launch[tb][tk];
    if (v >= 1 && v <= kNumKfWidths) return g_launch_kf[v - 1][tb][tk];
    return nullptr;
}

static void eri_register()
{
    register_eri_classes_a(g_launch);
    register_eri_kf_a(g_launch_kf);
    register_eri_kf_b(g_launch_kf);
    register_eri_kf_c(g_launch_kf);
    register_eri_kf_d(g_launch_kf);
    // default before tuning: the narrowest ket-first kernel built, else the team kernel
    for (int tb = 0; tb < kNumPairTypes; ++tb)
        for (int tk = 0; tk <= tb; ++tk) {
            g_variant[tb][tk] = 0;
            for (int v = kNumKfWidths; v >= 1; --v)
                if (variant_fn(tb, tk, v)) g_variant[tb][tk] = v;
        }
}

cudaError_t eri_module_init()
{
    static std::once_flag once;
    std::call_once(once, eri_register);
    return cudaSuccess;
}

int eri_num_variants() { return 1 + kNumKfWidths; }

int eri_variant(int tb, int tk)
{
    if (tb < 0 || tk < 0 || tb >= kNumPairTypes || tk >= kNumPairTypes || tb < tk) return -1;
    return g_variant[tb][tk];
}

int eri_set_variant(int tb, int tk, int variant)
{
    if (tb < 0 || tk < 0 || tb >= kNumPairTypes || tk >= kNumPairTypes || tb < tk) return -1;
    if (!variant_fn(tb, tk, variant)) return -1;
    g_variant[tb][tk] = variant;
    return 0;
}

cudaError_t eri_launch(int tb, int tk, const EriArgs& args, cudaStream_t st)
{
    if (tb < 0 || tk < 0 || tb >= kNumPairTypes || tk >= kNumPairTypes || tb < tk) return cudaErrorInvalidValue;
    variant_fn(tb, tk, g_variant[tb][tk])(args, st);
    count_launch();
    return cudaGetLastError();
}

cudaError_t pair_records_launch(const ShellPairDev* pairs, int npairs, const double* xyz, const int* poff,
                                const double* exps, const double* coefs, const int* plist, double* pp,
                                cudaStream_t st)
{
    if (npairs <= 0) return cudaSuccess;
    int blocks = npairs < 148 * 64 ? npairs : 148 * 64;
    k_pair_records<<<blocks, 64, 0, st>>>(pairs, npairs, xyz, poff, exps, coefs, plist, pp);
    count_launch();
    return cudaGetLastError();
}

cudaError_t boys_eval_launch(int m, int64_t n, const double* x, const double* table, double* out, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_boys_eval<<<(unsigned)blocks, 256, 0, st>>>(m, n, x, table, out);
    count_launch();
    return cudaGetLastError();
}

} // namespace gci
