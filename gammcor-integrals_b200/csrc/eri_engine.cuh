// eri_engine.cuh -- class-templated McMurchie-Davidson ERI kernel for sm_100a.
//
// One team of TW threads evaluates one contracted shell quartet (AB|CD) of a
// canonical class (LA>=LB, LC>=LD, bra type >= ket type).  The algorithm is
// the reference's (src/integrals/Auto2e): the (LS|KS) matrix
//   W(e,f) = sum_prims E^e_tuv (-1)^{tau+nu+phi} E^f R_{t+tau,u+nu,v+phi}
// with single-centre Hermite coefficients (auto2e_WMatrix_part1.f90:743-812),
// then the horizontal recurrence to (ab|cd) (auto2e_KetTransfer.f90) and the
// Cartesian -> spherical/normalisation transforms (auto2e_SpherTransf.f90,
// auto2e_Normalize_*).  The HRR is applied in its closed binomial form
//   (a, b| = sum_{k<=b} C(b,k) (A-B)^{b-k} (a+k, 0|
// so every output element is independent (no sequential recursion levels).
//
// Primitive-pair quantities (P, Rp, K_ab c_a c_b and the E^{e}_t tables) are
// precomputed once per shell pair (k_pair_records) and read through the
// read-only cache; R_tuv, the ket-transformed S(f,tuv) and the epilogue
// tensors live in shared memory; the W accumulator lives in registers, spread
// over the team's lanes.
#pragma once
#include "gci_common.h"
#include "boys.cuh"

namespace gci {

constexpr int kCartTab = cart_off(kMaxPairL + 3);   // levels 0..kMaxPairL+2
constexpr int kHermTab = herm_n(kMaxDerivLT);

struct DeviceTables {
    unsigned char cart[3 * kCartTab];
    unsigned char herm[3 * kHermTab];
    double binom[8][8];
};

// One copy per translation unit; filled by upload_device_tables() below.
static __constant__ DeviceTables c_tab;

static inline cudaError_t upload_device_tables()
{
    DeviceTables h{};
    for (int l = 0; l <= kMaxPairL + 2; ++l) {
        int i = cart_off(l);
        for (int x = l; x >= 0; --x)
            for (int y = l - x; y >= 0; --y) {
                h.cart[3 * i + 0] = (unsigned char)x;
                h.cart[3 * i + 1] = (unsigned char)y;
                h.cart[3 * i + 2] = (unsigned char)(l - x - y);
                ++i;
            }
    }
    for (int n = 0; n <= kMaxDerivLT; ++n)
        for (int s = 0; s <= n; ++s)
            for (int v = 0; v <= s; ++v) {
                int u = s - v, t = n - s;
                int i = herm_idx(t, u, v);
                h.herm[3 * i + 0] = (unsigned char)t;
                h.herm[3 * i + 1] = (unsigned char)u;
                h.herm[3 * i + 2] = (unsigned char)v;
            }
    for (int n = 0; n < 8; ++n)
        for (int k = 0; k < 8; ++k) {
            double b = 0.0;
            if (k <= n) { b = 1.0; for (int i = 0; i < k; ++i) b = b * (n - i) / (i + 1); }
            h.binom[n][k] = b;
        }
    return cudaMemcpyToSymbol(c_tab, &h, sizeof(h));
}

template <int TW, int TPB>
__device__ __forceinline__ void team_sync()
{
    if constexpr (TW == TPB && TPB > 32) {
        __syncthreads();
    } else if constexpr (TW == 32) {
        __syncwarp();
    } else if constexpr (TW > 1) {
        const unsigned lane_in_warp = threadIdx.x & 31u;
        const unsigned base = (lane_in_warp / TW) * TW;
        const unsigned mask = ((TW == 32) ? 0xffffffffu : ((1u << TW) - 1u)) << base;
        __syncwarp(mask);
    }
}

constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <int LA, int LB, int LC, int LD>
struct EriShape {
    static constexpr int L1 = LA + LB, L2 = LC + LD, LT = L1 + L2;
    static constexpr int E0 = cart_off(LA), NE = cart_off(L1 + 1) - E0;
    static constexpr int F0 = cart_off(LC), NF = cart_off(L2 + 1) - F0;
    static constexpr int HT = herm_n(LT), H1 = herm_n(L1);
    static constexpr int nA = ncart(LA), nB = ncart(LB), nC = ncart(LC), nD = ncart(LD);
    static constexpr int RSA = pp_record(L1), RSB = pp_record(L2);
    static constexpr int SZ_MAIN = 2 * HT + NF * H1;
    static constexpr int SZ_P0 = cmax(NE * NF, cmax(NE * nC * nD, nA * nB * nC * nD));
    static constexpr int SZ_P1 = cmax(NE * nC * nD, nA * nB * nC * nD);
    static constexpr int SZ_TEAM = cmax(SZ_MAIN, SZ_P0 + SZ_P1);
};

// Shared-memory view of one team's scratch: AoS per team for TW > 1,
// interleaved (element-major) across teams for TW == 1 so that neighbouring
// threads touch neighbouring words.
template <int TW, int TPB, int SZ>
struct TeamMem {
    static constexpr int NT = TPB / TW;
    static constexpr int STRIDE = (TW == 1) ? NT : 1;
    static constexpr int TEAM_SZ = (TW == 1) ? 1 : (SZ | 1);
    double* base;
    __device__ __forceinline__ double& operator[](int k) const { return base[k * STRIDE]; }
    __device__ __forceinline__ TeamMem shifted(int k) const { return TeamMem{base + k * STRIDE}; }
    static constexpr size_t bytes() { return sizeof(double) * (size_t)((TW == 1) ? NT * SZ : NT * TEAM_SZ); }
};

__device__ __forceinline__ void set_err(int* err, int code)
{
    if (err) atomicCAS(err, 0, code);
}

template <int LA, int LB, int LC, int LD, int TW, int TPB>
__global__ void __launch_bounds__(TPB) k_eri_class(const EriArgs a)
{
    using S = EriShape<LA, LB, LC, LD>;
    using TM = TeamMem<TW, TPB, S::SZ_TEAM>;
    constexpr int NT = TPB / TW;
    constexpr int NWORK = S::NE * S::NF;
    constexpr int WPL = (NWORK + TW - 1) / TW;
    extern __shared__ double smem[];
    const int team = threadIdx.x / TW;
    const int lane = threadIdx.x % TW;
    const TM ts{smem + ((TW == 1) ? team : team * TM::TEAM_SZ)};

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
        const int nbp = pb.nprim1 * pb.nprim2;
        const int nkp = pk.nprim1 * pk.nprim2;

        double w[WPL];
#pragma unroll
        for (int i = 0; i < WPL; ++i) w[i] = 0.0;

        const TM RA = ts;
        const TM RB = ts.shifted(S::HT);
        const TM SS = ts.shifted(2 * S::HT);

        for (int kp = 0; kp < nkp; ++kp) {
            const double* __restrict__ K = rk + (size_t)kp * S::RSB;
            const double Q = __ldg(K + 0);
            const double qx = __ldg(K + 1), qy = __ldg(K + 2), qz = __ldg(K + 3);
            const double pcd = __ldg(K + 4);
            const double* __restrict__ Ecx = K + 8;
            const double* __restrict__ Ecy = Ecx + tri(S::L2);
            const double* __restrict__ Ecz = Ecy + tri(S::L2);
            for (int bp = 0; bp < nbp; ++bp) {
                const double* __restrict__ Bp = rb + (size_t)bp * S::RSA;
                const double P = __ldg(Bp + 0);
                const double X = __ldg(Bp + 1) - qx, Y = __ldg(Bp + 2) - qy, Z = __ldg(Bp + 3) - qz;
                const double pab = __ldg(Bp + 4);
                const double PQ = P * Q;
                const double den = P + Q + a.kappa * PQ;
                const double alpha = PQ / den;
                // 2 pi^{5/2} / (PQ sqrt(P+Q+kappa PQ)) (auto2e_WMatrix_part1.f90:134)
                const double pref = 34.986836655249725 / (PQ * sqrt(den)) * pab * pcd;
                double F[S::LT + 1];
                boys_fm<S::LT>(alpha * (X * X + Y * Y + Z * Z), a.boys, F);
                {
                    double pw = pref;
                    const double m2a = -2.0 * alpha;
#pragma unroll
                    for (int m = 0; m <= S::LT; ++m) { F[m] *= pw; pw *= m2a; }
                }
                // ---- Hermite Coulomb integrals R^{(0)}_{tuv}, t+u+v <= LT ----
                TM cur = RA, nxt = RB;
                if (lane == 0) cur[0] = F[S::LT];
                team_sync<TW, TPB>();
#pragma unroll
                for (int j = S::LT - 1; j >= 0; --j) {
                    const int nent = herm_n(S::LT - j);
                    for (int h = lane; h < nent; h += TW) {
                        const int t = c_tab.herm[3 * h], u = c_tab.herm[3 * h + 1], v = c_tab.herm[3 * h + 2];
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
                    TM tmp = cur; cur = nxt; nxt = tmp;
                }
                // ---- ket Hermite -> Cartesian: S(f, tuv), tuv in bra range ----
                for (int idx = lane; idx < S::NF * S::H1; idx += TW) {
                    const int f = idx / S::H1, h = idx - f * S::H1;
                    const int fg = S::F0 + f;
                    const int fx = c_tab.cart[3 * fg], fy = c_tab.cart[3 * fg + 1], fz = c_tab.cart[3 * fg + 2];
                    const int t = c_tab.herm[3 * h], u = c_tab.herm[3 * h + 1], v = c_tab.herm[3 * h + 2];
                    double acc = 0.0;
                    for (int p3 = 0; p3 <= fz; ++p3) {
                        const double ez = __ldg(Ecz + fz * (fz + 1) / 2 + p3) * ((p3 & 1) ? -1.0 : 1.0);
                        double a2 = 0.0;
                        for (int p2 = 0; p2 <= fy; ++p2) {
                            const double ey = __ldg(Ecy + fy * (fy + 1) / 2 + p2) * ((p2 & 1) ? -1.0 : 1.0);
                            double a1 = 0.0;
                            for (int p1 = 0; p1 <= fx; ++p1) {
                                const double ex = __ldg(Ecx + fx * (fx + 1) / 2 + p1) * ((p1 & 1) ? -1.0 : 1.0);
                                a1 += ex * cur[herm_idx(t + p1, u + p2, v + p3)];
                            }
                            a2 += ey * a1;
                        }
                        acc += ez * a2;
                    }
                    SS[idx] = acc;
                }
                team_sync<TW, TPB>();
                // ---- bra Hermite -> Cartesian, accumulate W(e,f) ----
                const double* __restrict__ Ebx = Bp + 8;
                const double* __restrict__ Eby = Ebx + tri(S::L1);
                const double* __restrict__ Ebz = Eby + tri(S::L1);
#pragma unroll
                for (int i = 0; i < WPL; ++i) {
                    const int idx = lane + i * TW;
                    if (idx < NWORK) {
                        const int e = idx / S::NF, f = idx - e * S::NF;
                        const int eg = S::E0 + e;
                        const int ex = c_tab.cart[3 * eg], ey = c_tab.cart[3 * eg + 1], ez = c_tab.cart[3 * eg + 2];
                        const TM Sf = SS.shifted(f * S::H1);
                        double acc = 0.0;
                        for (int v = 0; v <= ez; ++v) {
                            double a2 = 0.0;
                            for (int u = 0; u <= ey; ++u) {
                                double a1 = 0.0;
                                for (int t = 0; t <= ex; ++t)
                                    a1 += __ldg(Ebx + ex * (ex + 1) / 2 + t) * Sf[herm_idx(t, u, v)];
                                a2 += __ldg(Eby + ey * (ey + 1) / 2 + u) * a1;
                            }
                            acc += __ldg(Ebz + ez * (ez + 1) / 2 + v) * a2;
                        }
                        w[i] += acc;
                    }
                }
                team_sync<TW, TPB>();
            }
        }

        // ================= epilogue: HRR + transforms + scatter =================
        const TM P0 = ts;
        const TM P1 = ts.shifted(S::SZ_P0);
#pragma unroll
        for (int i = 0; i < WPL; ++i) {
            const int idx = lane + i * TW;
            if (idx < NWORK) P0[idx] = w[i];
        }
        const int A = pb.s1, B = pb.s2, C = pk.s1, D = pk.s2;
        const double ABx = __ldg(a.sh_xyz + 3 * A) - __ldg(a.sh_xyz + 3 * B);
        const double ABy = __ldg(a.sh_xyz + 3 * A + 1) - __ldg(a.sh_xyz + 3 * B + 1);
        const double ABz = __ldg(a.sh_xyz + 3 * A + 2) - __ldg(a.sh_xyz + 3 * B + 2);
        const double CDx = __ldg(a.sh_xyz + 3 * C) - __ldg(a.sh_xyz + 3 * D);
        const double CDy = __ldg(a.sh_xyz + 3 * C + 1) - __ldg(a.sh_xyz + 3 * D + 1);
        const double CDz = __ldg(a.sh_xyz + 3 * C + 2) - __ldg(a.sh_xyz + 3 * D + 2);
        const int nfA = __ldg(a.sh_nfunc + A), nfB = __ldg(a.sh_nfunc + B);
        const int nfC = __ldg(a.sh_nfunc + C), nfD = __ldg(a.sh_nfunc + D);
        team_sync<TW, TPB>();
        // 1) ket HRR: X[e][c][d] (P1)
        for (int idx = lane; idx < S::NE * S::nC * S::nD; idx += TW) {
            const int e = idx / (S::nC * S::nD);
            const int r = idx - e * (S::nC * S::nD);
            const int c = r / S::nD, d = r - c * S::nD;
            const int cg = cart_off(LC) + c, dg = cart_off(LD) + d;
            const int cx = c_tab.cart[3 * cg], cy = c_tab.cart[3 * cg + 1], cz = c_tab.cart[3 * cg + 2];
            const int dx = c_tab.cart[3 * dg], dy = c_tab.cart[3 * dg + 1], dz = c_tab.cart[3 * dg + 2];
            double acc = 0.0;
            double pz = 1.0;
            for (int kz = dz; kz >= 0; --kz) {
                double py = 1.0;
                for (int ky = dy; ky >= 0; --ky) {
                    double px = 1.0;
                    for (int kx = dx; kx >= 0; --kx) {
                        const int lev = LC + kx + ky + kz;
                        const int fi = cart_off(lev) + cart_pos(cy + ky, cz + kz) - S::F0;
                        acc += c_tab.binom[dx][kx] * c_tab.binom[dy][ky] * c_tab.binom[dz][kz] * px * py * pz *
                               P0[e * S::NF + fi];
                        px *= CDx;
                    }
                    py *= CDy;
                }
                pz *= CDz;
            }
            P1[idx] = acc;
        }
        team_sync<TW, TPB>();
        // 2) T_D on d: U[e][c][md] (P0)
        const double* __restrict__ TA = a.tmat + __ldg(a.sh_toff + A);
        const double* __restrict__ TB = a.tmat + __ldg(a.sh_toff + B);
        const double* __restrict__ TC = a.tmat + __ldg(a.sh_toff + C);
        const double* __restrict__ TD = a.tmat + __ldg(a.sh_toff + D);
        for (int idx = lane; idx < S::NE * S::nC * nfD; idx += TW) {
            const int ec = idx / nfD, md = idx - ec * nfD;
            double acc = 0.0;
#pragma unroll
            for (int d = 0; d < S::nD; ++d) acc += __ldg(TD + md * S::nD + d) * P1[ec * S::nD + d];
            P0[idx] = acc;
        }
        team_sync<TW, TPB>();
        // 3) T_C on c: Y[e][mc][md] (P1)
        const int nq = nfC * nfD;
        for (int idx = lane; idx < S::NE * nq; idx += TW) {
            const int e = idx / nq, q = idx - e * nq;
            const int mc = q / nfD, md = q - mc * nfD;
            double acc = 0.0;
#pragma unroll
            for (int c = 0; c < S::nC; ++c)
                acc += __ldg(TC + mc * S::nC + c) * P0[(e * S::nC + c) * nfD + md];
            P1[idx] = acc;
        }
        team_sync<TW, TPB>();
        // 4) bra HRR: Z[a][b][q] (P0)
        for (int idx = lane; idx < S::nA * S::nB * nq; idx += TW) {
            const int ab = idx / nq, q = idx - ab * nq;
            const int ai = ab / S::nB, bi = ab - ai * S::nB;
            const int ag = cart_off(LA) + ai, bg = cart_off(LB) + bi;
            const int ax = c_tab.cart[3 * ag], ay = c_tab.cart[3 * ag + 1], az = c_tab.cart[3 * ag + 2];
            const int bx = c_tab.cart[3 * bg], by = c_tab.cart[3 * bg + 1], bz = c_tab.cart[3 * bg + 2];
            double acc = 0.0;
            double pz = 1.0;
            for (int kz = bz; kz >= 0; --kz) {
                double py = 1.0;
                for (int ky = by; ky >= 0; --ky) {
                    double px = 1.0;
                    for (int kx = bx; kx >= 0; --kx) {
                        const int lev = LA + kx + ky + kz;
                        const int ei = cart_off(lev) + cart_pos(ay + ky, az + kz) - S::E0;
                        acc += c_tab.binom[bx][kx] * c_tab.binom[by][ky] * c_tab.binom[bz][kz] * px * py * pz *
                               P1[ei * nq + q];
                        px *= ABx;
                    }
                    py *= ABy;
                }
                pz *= ABz;
            }
            P0[idx] = acc;
        }
        team_sync<TW, TPB>();
        // 5) T_B on b: V1[a][mb][q] (P1)
        for (int idx = lane; idx < S::nA * nfB * nq; idx += TW) {
            const int am = idx / nq, q = idx - am * nq;
            const int ai = am / nfB, mb = am - ai * nfB;
            double acc = 0.0;
#pragma unroll
            for (int b = 0; b < S::nB; ++b) acc += __ldg(TB + mb * S::nB + b) * P0[(ai * S::nB + b) * nq + q];
            P1[idx] = acc;
        }
        team_sync<TW, TPB>();
        // 6) T_A on a and scatter
        const ShellPairDev& pbr = pb;
        const ShellPairDev& pkr = pk;
        const int nout = nfA * nfB * nq;
        for (int idx = lane; idx < nout; idx += TW) {
            const int mm = idx / nq, q = idx - mm * nq;
            const int ma = mm / nfB, mb = mm - ma * nfB;
            const int mc = q / nfD, md = q - mc * nfD;
            double val = 0.0;
#pragma unroll
            for (int ai = 0; ai < S::nA; ++ai) val += __ldg(TA + ma * S::nA + ai) * P1[(ai * nfB + mb) * nq + q];
            // canonical -> stored orientation of each pair
            const int fb = pbr.swap ? (mb + nfB * ma) : (ma + nfA * mb);
            const int fk = pkr.swap ? (md + nfD * mc) : (mc + nfC * md);
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
                // dense symmetric AO-pair layout [p][q][j], the stored bra pair gives (p,q)
                const ShellPairDev& ps = a.swap_bk ? pkr : pbr;
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
        team_sync<TW, TPB>();
    }
}

} // namespace gci
