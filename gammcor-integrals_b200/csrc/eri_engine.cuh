// eri_engine.cuh -- class-templated McMurchie-Davidson ERI kernel for sm_100a.
//
// One team of TW threads evaluates one contracted shell quartet (AB|CD) of a
// canonical class (LA>=LB, LC>=LD, bra type >= ket type).  The integral is the
// reference's (src/integrals/Auto2e) Hermite-Coulomb sum
//   (ab|cd) = sum_prims E^{ab}_tuv (-1)^{tau+nu+phi} E^{cd}_{tau nu phi} R_{t+tau,u+nu,v+phi}
// followed by the Cartesian -> spherical / normalisation transforms
// (auto2e_SpherTransf.f90, auto2e_Normalize_*).  Unlike the reference, which
// contracts single-centre (e0|f0) and then applies the horizontal recurrence
// (auto2e_KetTransfer.f90), the bra and ket use two-centre coefficients E^{ab}
// per primitive pair: the recurrence after contraction cancels
// catastrophically when a contracted shell mixes tight and diffuse primitives
// on distant centres (all digits of (ff|ff) lost for exponents in
// [0.05, 5e3] 4.6 bohr apart), while the two-centre coefficients carry no
// such cancellation.  The sums are reordered for the GPU:
//
//  * for each ket primitive pair k, the bra side is contracted over all bra
//    primitive pairs i in Hermite space first:
//        T(ab, g) = sum_i sum_{h in supp(ab)} Eb_i(ab, h) R_ik(h + g)
//    with lane g of the team owning the ket Hermite index g = (tau,nu,phi)
//    and T(ab, g) for every bra Cartesian pair in registers;
//  * the ket transform W(ab, cd) += sum_g (-1)^|g| Ek_k(cd, g) T(ab, g) then
//    runs once per ket primitive pair instead of once per primitive quartet;
//  * the epilogue applies the four one-index transforms and scatters.
//
// R_tuv (Helgaker 9.9.18-20), the bra coefficient products and W live in
// shared memory; all index tables are built in shared memory once per block.
#pragma once
#include "gci_common.h"
#include "boys.cuh"

namespace gci {

template <int LA, int LB, int LC, int LD>
struct EriShape {
    static constexpr int L1 = LA + LB, L2 = LC + LD, LT = L1 + L2;
    static constexpr int nA = ncart(LA), nB = ncart(LB), nC = ncart(LC), nD = ncart(LD);
    static constexpr int NE = nA * nB, NF = nC * nD;     // bra (a,b) and ket (c,d) Cartesian pairs
    static constexpr int HT = herm_n(LT), H1 = herm_n(L1), H2 = herm_n(L2);
    static constexpr int EA = e2_size(LA, LB), EC = e2_size(LC, LD);   // per-axis coefficient tables
    static constexpr int RSA = pp_record(LA, LB), RSB = pp_record(LC, LD);
    static constexpr int POA = pp_prod_off(LA, LB), POC = pp_prod_off(LC, LD);   // product tables
    static constexpr int NCB = pair_ncb(LA, LB), NCK = pair_ncb(LC, LD);
    // team scratch (doubles): W, R ping-pong, T spill
    static constexpr int O_W = 0, O_RA = NE * NF, O_RB = O_RA + HT, O_TT = O_RB + HT;
    static constexpr int SZ_MAIN = O_TT + NE * H2;
    // epilogue ping-pong over the same scratch (P0 holds W on entry); every
    // stage has at most NE * NF elements (spherical counts <= Cartesian)
    static constexpr int SZ_P0 = NE * NF, SZ_P1 = NE * NF;
    static constexpr int SZ_TEAM = cmax(SZ_MAIN, SZ_P0 + SZ_P1);
    // per-block tables (ints)
    static constexpr int TAB_RIDX = H2 * H1;      // R index of h + g
    static constexpr int TAB_HERM = HT;           // packed (t,u,v) of each Hermite index
    static constexpr int TAB_INTS = TAB_RIDX + TAB_HERM;
};

// Team geometry: TW lanes own the ket Hermite indices (TW >= H2).  Teams of at
// most 32 lanes are packed floor(32/TW) per warp in one-warp blocks; wider
// teams fill a block of their own.
template <int LA, int LB, int LC, int LD>
struct EriTeam {
    using S = EriShape<LA, LB, LC, LD>;
    static constexpr int TW = S::H2 <= 32 ? S::H2 : 32 * ((S::H2 + 31) / 32);
    static constexpr int TPB = TW <= 32 ? 32 : TW;
    static constexpr int TEAM_SZ = S::SZ_TEAM | 1;
    // teams per block: as many as fit in a warp, within ~96 KB of team scratch
    static constexpr int NT_WARP = TW <= 32 ? 32 / TW : 1;
    static constexpr int NT_SMEM = (int)((96 * 1024) / (sizeof(double) * TEAM_SZ));
    static constexpr int NT = NT_WARP < NT_SMEM ? NT_WARP : (NT_SMEM > 0 ? NT_SMEM : 1);
    static constexpr size_t smem_bytes()
    {
        return sizeof(double) * (size_t)NT * TEAM_SZ + sizeof(int) * (size_t)S::TAB_INTS;
    }
};

template <int TW, int TPB>
__device__ __forceinline__ void team_sync()
{
    if constexpr (TW > 32) {
        __syncthreads();
    } else if constexpr (TW == 32) {
        __syncwarp();
    } else if constexpr (TW > 1) {
        const unsigned base = (threadIdx.x / TW) * TW;
        __syncwarp(((1u << TW) - 1u) << base);
    }
}

__device__ __forceinline__ void set_err(int* err, int code)
{
    if (err) atomicCAS(err, 0, code);
}

// Epilogue of one quartet: the four one-index transforms T_D, T_C, T_B, T_A
// (normalisation and Cartesian -> spherical) of W[ab][cd] held in P0, and the
// scatter into the output through the row/column maps.  P1 is scratch of
// NE * NF doubles; lanes of the team share the work.
template <int LA, int LB, int LC, int LD, int TW, int TPB>
__device__ __forceinline__ void eri_epilogue(const EriArgs& a, const ShellPairDev& pb, const ShellPairDev& pk,
                                             int bra, int ket, double* P0, double* P1, int lane)
{
    using S = EriShape<LA, LB, LC, LD>;
    const int A = pb.s1, B = pb.s2, C = pk.s1, D = pk.s2;
    const int nfA = __ldg(a.sh_nfunc + A), nfB = __ldg(a.sh_nfunc + B);
    const int nfC = __ldg(a.sh_nfunc + C), nfD = __ldg(a.sh_nfunc + D);
    const double* __restrict__ TA = a.tmat + __ldg(a.sh_toff + A);
    const double* __restrict__ TB = a.tmat + __ldg(a.sh_toff + B);
    const double* __restrict__ TC = a.tmat + __ldg(a.sh_toff + C);
    const double* __restrict__ TD = a.tmat + __ldg(a.sh_toff + D);
    // 1) T_D on d: U[ab][c][md] (P1)
    for (int idx = lane; idx < S::NE * S::nC * nfD; idx += TW) {
        const int ec = idx / nfD, md = idx - ec * nfD;
        double acc = 0.0;
#pragma unroll
        for (int d = 0; d < S::nD; ++d) acc += __ldg(TD + md * S::nD + d) * P0[ec * S::nD + d];
        P1[idx] = acc;
    }
    team_sync<TW, TPB>();
    // 2) T_C on c: Y[ab][mc][md] (P0)
    const int nq = nfC * nfD;
    for (int idx = lane; idx < S::NE * nq; idx += TW) {
        const int e = idx / nq, q = idx - e * nq;
        const int mc = q / nfD, md = q - mc * nfD;
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < S::nC; ++c) acc += __ldg(TC + mc * S::nC + c) * P1[(e * S::nC + c) * nfD + md];
        P0[idx] = acc;
    }
    team_sync<TW, TPB>();
    // 3) T_B on b: V1[a][mb][q] (P1)
    for (int idx = lane; idx < S::nA * nfB * nq; idx += TW) {
        const int am = idx / nq, q = idx - am * nq;
        const int ai = am / nfB, mb = am - ai * nfB;
        double acc = 0.0;
#pragma unroll
        for (int b = 0; b < S::nB; ++b) acc += __ldg(TB + mb * S::nB + b) * P0[(ai * S::nB + b) * nq + q];
        P1[idx] = acc;
    }
    team_sync<TW, TPB>();
    // 4) T_A on a and scatter
    const int nout = nfA * nfB * nq;
    for (int idx = lane; idx < nout; idx += TW) {
        const int mm = idx / nq, q = idx - mm * nq;
        const int ma = mm / nfB, mb = mm - ma * nfB;
        const int mc = q / nfD, md = q - mc * nfD;
        double val = 0.0;
#pragma unroll
        for (int ai = 0; ai < S::nA; ++ai) val += __ldg(TA + ma * S::nA + ai) * P1[(ai * nfB + mb) * nq + q];
        // canonical -> stored orientation of each pair
        const int fb = pb.swap ? (mb + nfB * ma) : (ma + nfA * mb);
        const int fk = pk.swap ? (md + nfD * mc) : (mc + nfC * md);
        const int rowf = a.swap_bk ? fk : fb;
        const int colf = a.swap_bk ? fb : fk;
        if (a.mode == kModeProduct) {
            const int row = a.row_map[a.row_off[bra] + rowf];
            const int col = a.col_map[a.col_off[ket] + colf];
            if (row >= 0 && col >= 0) a.out[row + a.ldo * (int64_t)col] = val;
        } else if (a.mode == kModeDiagonal) {
            if (rowf == colf) {
                const int row = a.row_map[a.row_off[bra] + rowf];
                if (row >= 0) a.out[row] = val;
            }
        } else {
            // dense symmetric AO-pair layout [p][q][j]; the stored bra pair gives (p, q)
            const ShellPairDev& ps = a.swap_bk ? pk : pb;
            const int first = ps.swap ? ps.s2 : ps.s1;
            const int second = ps.swap ? ps.s1 : ps.s2;
            const int n1 = __ldg(a.sh_nfunc + first);
            const int i1 = rowf % n1, i2 = rowf / n1;
            const int j = a.col_map[a.col_off[ket] + colf];
            if (j >= 0) {
                const int64_t p = __ldg(a.sh_loc + first) + i1, qq = __ldg(a.sh_loc + second) + i2;
                a.out[(p * a.nao + qq) * a.jcount + j] = val;
                if (first != second) a.out[(qq * a.nao + p) * a.jcount + j] = val;
            }
        }
    }
}

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(EriTeam<LA, LB, LC, LD>::TPB)
k_eri_class(const EriArgs a)
{
    using S = EriShape<LA, LB, LC, LD>;
    using G = EriTeam<LA, LB, LC, LD>;
    constexpr int TW = G::TW, TPB = G::TPB, NT = G::NT;
    extern __shared__ double smem[];
    int* tab = reinterpret_cast<int*>(smem + (size_t)NT * G::TEAM_SZ);
    int* tab_ridx = tab;                     // [g][h] -> herm_idx(h + g)
    int* tab_herm = tab_ridx + S::TAB_RIDX;  // t | u << 8 | v << 16

    // ---- per-block tables
    for (int c = threadIdx.x; c < S::TAB_RIDX; c += TPB) {
        const int g = c / S::H1, h = c - g * S::H1;
        tab_ridx[c] = herm_idx(herm_t(h) + herm_t(g), herm_u(h) + herm_u(g), herm_v(h) + herm_v(g));
    }
    for (int c = threadIdx.x; c < S::HT; c += TPB) tab_herm[c] = herm_t(c) | (herm_u(c) << 8) | (herm_v(c) << 16);
    __syncthreads();

    const int team = threadIdx.x / TW;
    const int lane = threadIdx.x - team * TW;
    if (team >= NT) return;   // lanes left over when TW does not divide 32
    double* ts = smem + (size_t)team * G::TEAM_SZ;
    double* RA = ts + S::O_RA;
    double* RB = ts + S::O_RB;
    double* TT = ts + S::O_TT;
    double* WW = ts + S::O_W;

    const int64_t ntasks = (a.mode == kModeDiagonal) ? a.nbra : a.nbra * a.nket;
    const int64_t stride = (int64_t)gridDim.x * NT;
    for (int64_t task = (int64_t)blockIdx.x * NT + team; task < ntasks; task += stride) {
        int bra, ket;
        if (a.mode == kModeDiagonal) {
            bra = ket = a.bra_ids[task];
        } else {
            bra = a.bra_ids[task % a.nbra];
            ket = a.ket_ids[task / a.nbra];
        }
        const int cb = a.swap_bk ? ket : bra;
        const int ck = a.swap_bk ? bra : ket;
        const ShellPairDev pb = a.pairs[cb];
        const ShellPairDev pk = a.pairs[ck];
        const double* __restrict__ rb = a.pp + pb.rec_off;
        const double* __restrict__ rk = a.pp + pk.rec_off;
        const int nbp = pb.npp;
        const int nkp = pk.npp;

        for (int w = lane; w < S::NE * S::NF; w += TW) WW[w] = 0.0;
        // lane -> ket Hermite index g and the R indices it reads
        const bool gl = lane < S::H2;
        const int* ridx = tab_ridx + (gl ? lane : 0) * S::H1;

        for (int kp = 0; kp < nkp; ++kp) {
            const double* __restrict__ K = rk + (size_t)kp * S::RSB;
            const double Q = __ldg(K + 0);
            const double qx = __ldg(K + 1), qy = __ldg(K + 2), qz = __ldg(K + 3);
            const double pcd = __ldg(K + 4);
            double T[S::NE];
#pragma unroll
            for (int e = 0; e < S::NE; ++e) T[e] = 0.0;

            for (int bp = 0; bp < nbp; ++bp) {
                const double* __restrict__ Bp = rb + (size_t)bp * S::RSA;
                const double P = __ldg(Bp + 0);
                const double X = __ldg(Bp + 1) - qx, Y = __ldg(Bp + 2) - qy, Z = __ldg(Bp + 3) - qz;
                const double PQ = P * Q;
                const double den = P + Q + a.kappa * PQ;
                const double alpha = PQ / den;
                // 2 pi^{5/2} / (PQ sqrt(P+Q+kappa PQ)) (auto2e_WMatrix_part1.f90:134)
                const double pref = 34.986836655249725 / (PQ * sqrt(den)) * __ldg(Bp + 4) * pcd;
                double F[S::LT + 1];
                boys_fm<S::LT>(alpha * (X * X + Y * Y + Z * Z), a.boys, F);
                {
                    double pw = pref;
                    const double m2a = -2.0 * alpha;
#pragma unroll
                    for (int m = 0; m <= S::LT; ++m) { F[m] *= pw; pw *= m2a; }
                }
                // bra coefficient products Eb(ab, h) of this bra primitive pair
                const double* __restrict__ CBv = Bp + S::POA;
                // Hermite Coulomb integrals R^{(0)}_{tuv}, t+u+v <= LT
                double* cur = RA;
                double* nxt = RB;
                if (lane == 0) cur[0] = F[S::LT];
                team_sync<TW, TPB>();
#pragma unroll
                for (int j = S::LT - 1; j >= 0; --j) {
                    const int nent = herm_n(S::LT - j);
                    for (int h = lane; h < nent; h += TW) {
                        const int p = tab_herm[h];
                        const int t = p & 0xff, u = (p >> 8) & 0xff, v = p >> 16;
                        double r;
                        if (t > 0) {
                            r = X * cur[herm_idx(t - 1, u, v)];
                            if (t > 1) r += (double)(t - 1) * cur[herm_idx(t - 2, u, v)];
                        } else if (u > 0) {
                            r = Y * cur[herm_idx(t, u - 1, v)];
                            if (u > 1) r += (double)(u - 1) * cur[herm_idx(t, u - 2, v)];
                        } else if (v > 0) {
                            r = Z * cur[herm_idx(t, u, v - 1)];
                            if (v > 1) r += (double)(v - 1) * cur[herm_idx(t, u, v - 2)];
                        } else {
                            r = F[j];
                        }
                        nxt[h] = r;
                    }
                    team_sync<TW, TPB>();
                    double* tmp = cur; cur = nxt; nxt = tmp;
                }
                // T(e, g) += sum_{h in supp(e)} Eb(e, h) R(h + g)
                if (gl) {
                    if constexpr (S::H1 <= 56) {
                        double Rl[S::H1];
#pragma unroll
                        for (int h = 0; h < S::H1; ++h) Rl[h] = cur[ridx[h]];
                        int c = 0;
#pragma unroll
                        for (int e = 0; e < S::NE; ++e) {
                            double acc = T[e];
#pragma unroll
                            for (int v = 0; v <= pair_z(LA, LB, e); ++v)
#pragma unroll
                                for (int u = 0; u <= pair_y(LA, LB, e); ++u)
#pragma unroll
                                    for (int t = 0; t <= pair_x(LA, LB, e); ++t) {
                                        acc += __ldg(CBv + c) * Rl[herm_idx(t, u, v)];
                                        ++c;
                                    }
                            T[e] = acc;
                        }
                    } else {
                        int c = 0;
#pragma unroll
                        for (int e = 0; e < S::NE; ++e) {
                            double acc = T[e];
#pragma unroll
                            for (int v = 0; v <= pair_z(LA, LB, e); ++v)
#pragma unroll
                                for (int u = 0; u <= pair_y(LA, LB, e); ++u)
#pragma unroll
                                    for (int t = 0; t <= pair_x(LA, LB, e); ++t) {
                                        acc += __ldg(CBv + c) * cur[ridx[herm_idx(t, u, v)]];
                                        ++c;
                                    }
                            T[e] = acc;
                        }
                    }
                }
                team_sync<TW, TPB>();
            }
            // ---- ket transform for this ket primitive pair:
            //      W(e, f) += sum_{g in supp(f)} (-1)^{tau+nu+phi} Ek(f, g) T(e, g)
            if (gl) {
#pragma unroll
                for (int e = 0; e < S::NE; ++e) TT[e * S::H2 + lane] = T[e];
            }
            team_sync<TW, TPB>();
            {
                const double* __restrict__ Ekx = K + 8;
                const double* __restrict__ Eky = Ekx + S::EC;
                const double* __restrict__ Ekz = Eky + S::EC;
                for (int f = lane; f < S::NF; f += TW) {
                    const int fx = pair_x(LC, LD, f), fy = pair_y(LC, LD, f), fz = pair_z(LC, LD, f);
                    const int ox = pair_ox(LC, LD, f), oy = pair_oy(LC, LD, f), oz = pair_oz(LC, LD, f);
                    double wcol[S::NE];
#pragma unroll
                    for (int e = 0; e < S::NE; ++e) wcol[e] = WW[e * S::NF + f];
                    for (int p3 = 0; p3 <= fz; ++p3) {
                        const double cz = __ldg(Ekz + oz + p3) * ((p3 & 1) ? -1.0 : 1.0);
                        for (int p2 = 0; p2 <= fy; ++p2) {
                            const double cyz = cz * __ldg(Eky + oy + p2) * ((p2 & 1) ? -1.0 : 1.0);
                            for (int p1 = 0; p1 <= fx; ++p1) {
                                const double c = cyz * __ldg(Ekx + ox + p1) * ((p1 & 1) ? -1.0 : 1.0);
                                const int g = herm_idx(p1, p2, p3);
#pragma unroll
                                for (int e = 0; e < S::NE; ++e) wcol[e] += c * TT[e * S::H2 + g];
                            }
                        }
                    }
#pragma unroll
                    for (int e = 0; e < S::NE; ++e) WW[e * S::NF + f] = wcol[e];
                }
            }
            team_sync<TW, TPB>();
        }

        // ================= epilogue: transforms + scatter =================
        eri_epilogue<LA, LB, LC, LD, TW, TPB>(a, pb, pk, bra, ket, WW, WW + S::SZ_P0, lane);
        team_sync<TW, TPB>();
    }
}

} // namespace gci
