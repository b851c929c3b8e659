// grad_engine.cuh -- Coulomb energy, nuclear gradient and Coulomb matrix of a
// density by McMurchie-Davidson Hermite index shifts: the adjoint of the ERI
// path.  The reference has no derivative integrals; the Hermite machinery is
// the one of its ERI engine (src/integrals/Auto2e: E coefficients
// auto2e_Hermite.f90:10-423, R_tuv :425-11878, prefactor
// auto2e_WMatrix_part1.f90:134).
//
// J = 1/2 sum_{pq,rs} D_pq (pq|rs) D_rs.  The density is contracted into
// Hermite space once per primitive pair i of a shell pair (A, B) (A >= B,
// first shell s1 of the canonical orientation on centre A):
//   h_i(t)    = w_AB K_i sum_ab Ds_ab E^{ab}_t                      t <= lA+lB
//   gA_i,x(t) = w_AB K_i sum_ab Ds_ab [2a E^{a+1x,b}_t - a_x E^{a-1x,b}_t]
//   gB_i,x(t) = w_AB K_i sum_ab Ds_ab [2b E^{a,b+1x}_t - b_x E^{a,b-1x}_t]   t <= lA+lB+1
// with w_AB = 2 for A != B (the pair stands for (A,B) and (B,A)), 1 for
// A == B, Ds = (D + D^T)/2 in Cartesian components (norms and the spherical
// transform folded in), K_i = exp(-ab/p |AB|^2) c_a c_b, and
// d/dA_x of a Cartesian Gaussian = 2a G_{a+1x} - a_x G_{a-1x}.  The
// potential of the whole density at pair i,
//   V_i(t) = sum_k 2 pi^{5/2} / (P Q sqrt(P+Q+kappa PQ)) sum_tau (-1)^|tau| h_k(tau) R_{t+tau}
// (the potential kernel below, t up to lA+lB+1) then gives
//   J          = 1/2 sum_i h_i . V_i
//   dJ/dA_x   += gA_i,x . V_i,   dJ/dB_x += gB_i,x . V_i
//   J_pq       = sum_i K_i sum_t E^{pq}_t V_i(t)   (Coulomb matrix, dJ/dD_pq)
// Only bra derivatives are needed: summed over all ordered (bra, ket) pairs,
// the ket derivatives of (pq|rs) are the bra derivatives of (rs|pq).
#pragma once
#include "gci_common.h"
#include "boys.cuh"
#include <type_traits>
#include <utility>

namespace gci {


// compile-time loop I = B .. N-1 (a fold expression: no recursion depth limit)
template <int B, class Fn, int... Is>
__device__ __forceinline__ void grad_static_for_impl(Fn& fn, std::integer_sequence<int, Is...>)
{
    (fn(std::integral_constant<int, B + Is>{}), ...);
}
template <int B, int N, class Fn>
__device__ __forceinline__ void grad_static_for(Fn&& fn)
{
    if constexpr (N > B) grad_static_for_impl<B>(fn, std::make_integer_sequence<int, N - B>{});
}

// R_tuv of one primitive quartet in registers, one array per Hermite level
// (a single array of more than ~200 doubles is demoted to local memory as a
// whole; per-level arrays keep the values in registers as far as they fit)
template <int L, int N, bool End = (L > N)>
struct RLevels : RLevels<L + 1, N> {
    double lv[tri(L)];
};
template <int L, int N>
struct RLevels<L, N, true> {
};
template <int H, int N>
__device__ __forceinline__ double& rget(RLevels<0, N>& R)
{
    constexpr int l = herm_level(H);
    constexpr int pos = H - (l > 0 ? herm_n(l - 1) : 0);
    return static_cast<RLevels<l, N>&>(R).lv[pos];
}

// One warp per (bra primitive pair, chunk of ket primitive pairs); each lane
// evaluates whole primitive quartets (Boys values, the R_tuv recursion in
// place, the ket contraction) and accumulates the potential V(t) in
// registers; the warp's sum is added to V once per chunk.
template <int L1, int L2>
__global__ void __launch_bounds__(128) k_grad_potential(const GradPotArgs a)
{
    constexpr int HB = grad_hb(L1), HK = herm_n(L2), N = L1 + 1 + L2;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= a.nbra * a.nchunk) return;   // uniform per warp
    const int64_t i = warp / a.nchunk, c = warp - i * a.nchunk;
    const int64_t gi = a.bra_beg + i;
    const double P = __ldg(a.mP + gi), px = __ldg(a.mX + gi), py = __ldg(a.mY + gi), pz = __ldg(a.mZ + gi);
    double Vacc[HB];
#pragma unroll
    for (int h = 0; h < HB; ++h) Vacc[h] = 0.0;
    const int64_t k0 = c * a.chunk;
    const int64_t k1 = k0 + a.chunk < a.nket ? k0 + a.chunk : a.nket;
    for (int64_t k = k0 + lane; k < k1; k += 32) {
        const int64_t gk = a.ket_beg + k;
        const double Q = __ldg(a.mP + gk);
        const double X = px - __ldg(a.mX + gk), Y = py - __ldg(a.mY + gk), Z = pz - __ldg(a.mZ + gk);
        const double PQ = P * Q, den = P + Q + a.kappa * PQ;
        const double alpha = PQ / den;
        const double pref = 2.0 * 17.49341832762486284626282167987155377876 / (PQ * sqrt(den));   // 2 pi^{5/2}
        double F[N + 1];
        boys_fm<N>(alpha * (X * X + Y * Y + Z * Z), a.boys, F);
        double Fs[N + 1];
        {
            double s = pref;
            const double m2a = -2.0 * alpha;
#pragma unroll
            for (int m = 0; m <= N; ++m) { Fs[m] = s * F[m]; s *= m2a; }
        }
        // R^{(j)}_{tuv} in place, order j = N .. 0: a level-l entry reads order j+1
        // at levels l-1 and l-2, so levels are updated from the top down and
        // R_000 last (Helgaker, Joergensen, Olsen 9.9.18-20)
        RLevels<0, N> R;
        rget<0, N>(R) = Fs[N];
        grad_static_for<0, N>([&](auto JJ) __attribute__((always_inline)) {
            constexpr int j = N - 1 - decltype(JJ)::value;
            constexpr int top = herm_n(N - j);
            grad_static_for<1, top>([&](auto HH) __attribute__((always_inline)) {
                constexpr int h = top - decltype(HH)::value;
                constexpr int t = herm_t(h), u = herm_u(h), v = herm_v(h);
                if constexpr (t > 0) {
                    double r = X * rget<herm_idx(t - 1, u, v), N>(R);
                    if constexpr (t > 1) r += (double)(t - 1) * rget<herm_idx(t - 2, u, v), N>(R);
                    rget<h, N>(R) = r;
                } else if constexpr (u > 0) {
                    double r = Y * rget<herm_idx(t, u - 1, v), N>(R);
                    if constexpr (u > 1) r += (double)(u - 1) * rget<herm_idx(t, u - 2, v), N>(R);
                    rget<h, N>(R) = r;
                } else {
                    double r = Z * rget<herm_idx(t, u, v - 1), N>(R);
                    if constexpr (v > 1) r += (double)(v - 1) * rget<herm_idx(t, u, v - 2), N>(R);
                    rget<h, N>(R) = r;
                }
            });
            rget<0, N>(R) = Fs[j];
        });
        // V(t) += sum_tau hk(tau) R(t + tau)
        grad_static_for<0, HK>([&](auto TT) __attribute__((always_inline)) {
            constexpr int g = decltype(TT)::value;
            constexpr int gt = herm_t(g), gu = herm_u(g), gv = herm_v(g);
            const double hv = __ldg(a.hk + (int64_t)g * a.nket + k);
            grad_static_for<0, HB>([&](auto HH) __attribute__((always_inline)) {
                constexpr int h = decltype(HH)::value;
                constexpr int r = herm_idx(herm_t(h) + gt, herm_u(h) + gu, herm_v(h) + gv);
                Vacc[h] = fma(hv, rget<r, N>(R), Vacc[h]);
            });
        });
    }
    double* Vi = a.V + i * HB;
#pragma unroll
    for (int h = 0; h < HB; ++h) {
        double s = Vacc[h];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == (h & 31)) atomicAdd(Vi + h, s);
    }
}

using GradLaunchFn = void (*)(const GradPotArgs&, cudaStream_t);
void register_grad_pot_a(GradLaunchFn (*tab)[kGradMaxL + 1]);
void register_grad_pot_b(GradLaunchFn (*tab)[kGradMaxL + 1]);
void register_grad_pot_c(GradLaunchFn (*tab)[kGradMaxL + 1]);

template <int L1, int L2>
static void launch_grad_potential(const GradPotArgs& a, cudaStream_t st)
{
    const int64_t warps = a.nbra * a.nchunk;
    const int64_t blocks = (warps + 3) / 4;
    k_grad_potential<L1, L2><<<(unsigned)blocks, 128, 0, st>>>(a);
}

// Classes (L1, L2) with L1 + L2 in [lo, hi] of bra levels L1 in [b0, b1].
template <int L1, int L2, int LO, int HI>
static void register_grad_one(GradLaunchFn (*tab)[kGradMaxL + 1])
{
    if constexpr (L1 + L2 >= LO && L1 + L2 <= HI) tab[L1][L2] = launch_grad_potential<L1, L2>;
}
template <int L1, int LO, int HI, int... K>
static void register_grad_row(GradLaunchFn (*tab)[kGradMaxL + 1], std::integer_sequence<int, K...>)
{
    (register_grad_one<L1, K, LO, HI>(tab), ...);
}
template <int LO, int HI, int... B>
static void register_grad_range(GradLaunchFn (*tab)[kGradMaxL + 1], std::integer_sequence<int, B...>)
{
    (register_grad_row<B, LO, HI>(tab, std::make_integer_sequence<int, kGradMaxL + 1>{}), ...);
}

} // namespace gci
