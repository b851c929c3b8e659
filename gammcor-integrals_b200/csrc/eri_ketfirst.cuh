// eri_ketfirst.cuh -- ket-first variant of the class kernels: the ket side is
// contracted inside the primitive loop and the bra side once per bra
// primitive pair.
//
// For a bra primitive pair i and the ket primitive pairs k of a quartet,
//   V_i(h, cd) = sum_k sum_{g in supp(cd)} (-1)^|g| Ek_k(cd, g) R_ik(h + g)
//   W(ab, cd) += sum_{h in supp(ab)} Eb_i(ab, h) V_i(h, cd)
// is the same Hermite-Coulomb sum as in eri_engine.cuh with the loops in the
// other order.  The work per primitive quartet is then H1 * (ket products)
// instead of (bra products) * H2, which for the bra-heavy classes that
// dominate Cholesky pivot columns ((ff|ss), (ff|ps), (fd|ss), ...) is smaller
// by one to two orders of magnitude; the bra products are applied once per
// bra primitive pair.
//
// A team of TW lanes (one warp, or a whole block of 64 or 128 threads)
// evaluates one quartet.  Lanes own bra Hermite
// indices h in the primitive loop (V in registers, the ket pairs cd taken in
// chunks that fit the register file; R is rebuilt per chunk) and elements of
// W in the bra update (registers when they fit, shared memory otherwise).
#pragma once
#include "eri_engine.cuh"
#include <type_traits>

namespace gci {

template <int I, int N, class Fn>
__device__ __forceinline__ void static_for(Fn&& fn)
{
    if constexpr (I < N) {
        fn(std::integral_constant<int, I>{});
        static_for<I + 1, N>(fn);
    }
}

// first ket product of Cartesian pair f in the product table of shells (lc, ld)
GCI_HD constexpr int pair_prod_off(int lc, int ld, int f)
{
    int n = 0;
    for (int i = 0; i < f; ++i) n += pair_supp(lc, ld, i);
    return n;
}

// Team width TWQ: one warp (several teams per block) or a whole block of 64
// or 128 threads per quartet; the autotuner picks the width per class.
template <int LA, int LB, int LC, int LD, int TWQ>
struct KfShape {
    using S = EriShape<LA, LB, LC, LD>;
    static constexpr int TW = TWQ;
    static constexpr int SLOTS = (S::H1 + TW - 1) / TW;        // bra Hermite indices per lane
    static constexpr int WSLOTS = (S::NE * S::NF + TW - 1) / TW;
    static constexpr bool WREG = WSLOTS <= 40;                 // W in registers, else shared memory
    // R(h + g) of a lane's bra Hermite indices held in registers (RL) or read
    // from shared memory per product (large ket classes)
    static constexpr bool RL = S::H2 <= 56;
    // ket pairs per chunk of the primitive loop: V (SLOTS x CH) and, with RL,
    // the lane's R values (H2) within ~88 doubles
    static constexpr int CH0 = RL ? (88 - S::H2) / SLOTS : 80 / SLOTS;
    static constexpr int CH = CH0 < 1 ? 1 : (CH0 > S::NF ? S::NF : CH0);
    static constexpr int NCH = (S::NF + CH - 1) / CH;
    // ket primitive pairs whose Boys values and geometry are prepared at once
    // (one per lane) and the stride of their entries: F_0..F_LT, X, Y, Z
    static constexpr int KB = 16, FS = S::LT + 4;
    // team scratch (doubles): R ping-pong, V and the prepared ket primitives
    // during the primitive loop; the epilogue's two buffers of NE*NF
    // afterwards (W in registers) or W kept apart from them (W in shared memory)
    static constexpr int O_RA = 0, O_RB = S::HT, O_V = 2 * S::HT, O_FK = O_V + S::H1 * S::NF;
    static constexpr int SZ_LOOP = O_FK + KB * FS;
    static constexpr int O_W = WREG ? 0 : cmax(SZ_LOOP, S::NE * S::NF);
    static constexpr int SZ = WREG ? cmax(SZ_LOOP, 2 * S::NE * S::NF) : O_W + S::NE * S::NF;
    // per-block tables: R recursion recipe of every Hermite index (its
    // coefficient as a double, then an int: source indices and axis); then
    // 16-bit entries (every value is below 2^15): R index of h + g, Hermite
    // index of every bra product, first bra product of each ab.  The 16-bit
    // tables and 16 prepared ket primitives keep the (f,f|f,d) block within
    // half of an SM's shared memory (two blocks per SM)
    static constexpr int TAB_INTS = S::HT;
    static constexpr int TAB_SHORTS = S::H2 * S::H1 + S::NCB + S::NE + 1;
    static_assert(S::HT < 32768 && S::NCB < 32768, "16-bit tables");
    // teams per block: four warps while their scratch stays within 160 KB
    static constexpr int TEAMS = TW > 32 ? 1
                                         : ((size_t)SZ * 8 * 4 <= 160 * 1024 ? 4
                                                                             : ((size_t)SZ * 8 * 2 <= 200 * 1024 ? 2 : 1));
    static constexpr int TPB = TW > 32 ? TW : 32 * TEAMS;
    static constexpr size_t smem_bytes()
    {
        return sizeof(double) * ((size_t)TEAMS * SZ + S::HT) + sizeof(int) * (size_t)TAB_INTS +
               sizeof(short) * (size_t)TAB_SHORTS;
    }
};

template <int LA, int LB, int LC, int LD, int TWQ>
__global__ void __launch_bounds__(KfShape<LA, LB, LC, LD, TWQ>::TPB)
k_eri_kf(const EriArgs a)
{
    using S = EriShape<LA, LB, LC, LD>;
    using K = KfShape<LA, LB, LC, LD, TWQ>;
    constexpr int TW = K::TW, TPB = K::TPB;
    extern __shared__ double smem[];
    double* tab_coef = smem + (size_t)K::TEAMS * K::SZ;           // recursion coefficient of h
    int* tab_rec = reinterpret_cast<int*>(tab_coef + S::HT);       // i1 | i2 << 12 | axis << 24
    short* tab_ridx = reinterpret_cast<short*>(tab_rec + S::HT);   // [g][h] -> herm_idx(h + g)
    short* tab_cbh = tab_ridx + S::H2 * S::H1;   // bra product -> Hermite index
    short* tab_cbo = tab_cbh + S::NCB;           // ab -> first bra product

    // R^{(j)}_{tuv} = d R^{(j+1)}_{tuv - e} + (n - 1) R^{(j+1)}_{tuv - 2e} along the first
    // nonzero axis e of (t,u,v) with component n (d = X, Y or Z); h = 0 takes F_j
    for (int c = threadIdx.x; c < S::HT; c += TPB) {
        const int t = herm_t(c), u = herm_u(c), v = herm_v(c);
        int ax = 3, i1 = 0, i2 = 0, n = 0;
        if (t > 0) { ax = 0; n = t; i1 = herm_idx(t - 1, u, v); i2 = t > 1 ? herm_idx(t - 2, u, v) : 0; }
        else if (u > 0) { ax = 1; n = u; i1 = herm_idx(t, u - 1, v); i2 = u > 1 ? herm_idx(t, u - 2, v) : 0; }
        else if (v > 0) { ax = 2; n = v; i1 = herm_idx(t, u, v - 1); i2 = v > 1 ? herm_idx(t, u, v - 2) : 0; }
        tab_rec[c] = i1 | (i2 << 12) | (ax << 24);
        tab_coef[c] = n > 1 ? (double)(n - 1) : 0.0;
    }
    for (int c = threadIdx.x; c < S::H2 * S::H1; c += TPB) {
        const int g = c / S::H1, h = c - g * S::H1;
        tab_ridx[c] = (short)herm_idx(herm_t(h) + herm_t(g), herm_u(h) + herm_u(g), herm_v(h) + herm_v(g));
    }
    for (int e = threadIdx.x; e < S::NE; e += TPB) {
        int off = 0;
        for (int f = 0; f < e; ++f) off += pair_supp(LA, LB, f);
        tab_cbo[e] = (short)off;
        const int ex = pair_x(LA, LB, e), ey = pair_y(LA, LB, e), ez = pair_z(LA, LB, e);
        for (int v = 0; v <= ez; ++v)
            for (int u = 0; u <= ey; ++u)
                for (int t = 0; t <= ex; ++t) tab_cbh[off++] = (short)herm_idx(t, u, v);
    }
    if (threadIdx.x == 0) tab_cbo[S::NE] = (short)S::NCB;
    __syncthreads();

    const int team = threadIdx.x / TW;
    const int lane = threadIdx.x - team * TW;
    double* ts = smem + (size_t)team * K::SZ;
    double* RA = ts + K::O_RA;
    double* RB = ts + K::O_RB;
    double* V = ts + K::O_V;
    double* Ws = ts + K::O_W;
    double* Fk = ts + K::O_FK;

    const int64_t ntasks = (a.mode == kModeDiagonal) ? a.nbra : a.nbra * a.nket;
    const int64_t stride = (int64_t)gridDim.x * K::TEAMS;
    for (int64_t task = (int64_t)blockIdx.x * K::TEAMS + team; task < ntasks; task += stride) {
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

        double Wr[K::WREG ? K::WSLOTS : 1];
        if constexpr (K::WREG) {
#pragma unroll
            for (int j = 0; j < K::WSLOTS; ++j) Wr[j] = 0.0;
        } else {
            for (int w = lane; w < S::NE * S::NF; w += TW) Ws[w] = 0.0;
        }

        for (int bp = 0; bp < nbp; ++bp) {
            const double* __restrict__ Bp = rb + (size_t)bp * S::RSA;
            const double P = __ldg(Bp + 0);
            const double px = __ldg(Bp + 1), py = __ldg(Bp + 2), pz = __ldg(Bp + 3);
            const double pab = __ldg(Bp + 4);

            static_for<0, K::NCH>([&](auto CI) {
                constexpr int f0 = decltype(CI)::value * K::CH;
                constexpr int f1 = (f0 + K::CH < S::NF) ? f0 + K::CH : S::NF;
                constexpr int c0 = pair_prod_off(LC, LD, f0);
                double Vr[K::SLOTS][K::CH];
#pragma unroll
                for (int s = 0; s < K::SLOTS; ++s)
#pragma unroll
                    for (int f = 0; f < K::CH; ++f) Vr[s][f] = 0.0;

                for (int k0 = 0; k0 < nkp; k0 += K::KB) {
                    const int kn = (nkp - k0) < K::KB ? (nkp - k0) : K::KB;
                    // Boys values (scaled by the prefactor and (-2 alpha)^m) and P - Q of
                    // this bra primitive with up to KB ket primitives, one per lane
                    for (int kk = lane; kk < kn; kk += TW) {
                        const double* __restrict__ Kp = rk + (size_t)(k0 + kk) * S::RSB;
                        const double Q = __ldg(Kp + 0);
                        const double X = px - __ldg(Kp + 1), Y = py - __ldg(Kp + 2), Z = pz - __ldg(Kp + 3);
                        const double PQ = P * Q;
                        const double den = P + Q + a.kappa * PQ;
                        const double alpha = PQ / den;
                        // 2 pi^{5/2} / (PQ sqrt(P+Q+kappa PQ)) (auto2e_WMatrix_part1.f90:134)
                        const double pref = 34.986836655249725 / (PQ * sqrt(den)) * pab * __ldg(Kp + 4);
                        double F[S::LT + 1];
                        boys_fm<S::LT>(alpha * (X * X + Y * Y + Z * Z), a.boys, F);
                        double* fk = Fk + kk * K::FS;
                        double pw = pref;
                        const double m2a = -2.0 * alpha;
#pragma unroll
                        for (int m = 0; m <= S::LT; ++m) { fk[m] = F[m] * pw; pw *= m2a; }
                        fk[S::LT + 1] = X; fk[S::LT + 2] = Y; fk[S::LT + 3] = Z;
                    }
                    team_sync<TW, TPB>();
                    for (int kk = 0; kk < kn; ++kk) {
                        const double* __restrict__ Kp = rk + (size_t)(k0 + kk) * S::RSB;
                        const double* fk = Fk + kk * K::FS;
                        const double X = fk[S::LT + 1], Y = fk[S::LT + 2], Z = fk[S::LT + 3];
                        // Hermite Coulomb integrals R^{(0)}_{tuv}, t+u+v <= LT (Helgaker 9.9.18-20)
                        double* cur = RA;
                        double* nxt = RB;
                        if (lane == 0) cur[0] = fk[S::LT];
                        team_sync<TW, TPB>();
#pragma unroll
                        for (int j = S::LT - 1; j >= 0; --j) {
                            const int nent = herm_n(S::LT - j);
                            const double Fj = fk[j];
                            for (int h = lane; h < nent; h += TW) {
                                const int rc = tab_rec[h];
                                const int ax = rc >> 24;
                                const double d = ax == 0 ? X : (ax == 1 ? Y : Z);
                                const double r = d * cur[rc & 0xfff] + tab_coef[h] * cur[(rc >> 12) & 0xfff];
                                nxt[h] = (h == 0) ? Fj : r;
                            }
                            team_sync<TW, TPB>();
                            double* tmp = cur; cur = nxt; nxt = tmp;
                        }
                        // V(h, cd) += sum_g (-1)^|g| Ek(cd, g) R(h + g), lane owns h = lane + TW s
                        const double* __restrict__ Ck = Kp + S::POC + c0;
#pragma unroll
                        for (int s = 0; s < K::SLOTS; ++s) {
                            const int h = lane + TW * s;
                            if (h < S::H1) {
                                double Rl[K::RL ? S::H2 : 1];
                                if constexpr (K::RL) {
#pragma unroll
                                    for (int g = 0; g < S::H2; ++g) Rl[g] = cur[tab_ridx[g * S::H1 + h]];
                                }
                                int c = 0;
#pragma unroll
                                for (int f = f0; f < f1; ++f) {
                                    double acc = Vr[s][f - f0];
#pragma unroll
                                    for (int v = 0; v <= pair_z(LC, LD, f); ++v)
#pragma unroll
                                        for (int u = 0; u <= pair_y(LC, LD, f); ++u)
#pragma unroll
                                            for (int t = 0; t <= pair_x(LC, LD, f); ++t) {
                                                const double e = __ldg(Ck + c);
                                                double rv;
                                                if constexpr (K::RL) rv = Rl[herm_idx(t, u, v)];
                                                else rv = cur[tab_ridx[herm_idx(t, u, v) * S::H1 + h]];
                                                if ((t + u + v) & 1) acc -= e * rv;
                                                else acc += e * rv;
                                                ++c;
                                            }
                                    Vr[s][f - f0] = acc;
                                }
                            }
                        }
                        team_sync<TW, TPB>();
                    }
                }
                // this chunk of V to shared memory
#pragma unroll
                for (int s = 0; s < K::SLOTS; ++s) {
                    const int h = lane + TW * s;
                    if (h < S::H1) {
#pragma unroll
                        for (int f = f0; f < f1; ++f) V[h * S::NF + f] = Vr[s][f - f0];
                    }
                }
            });
            team_sync<TW, TPB>();
            // W(ab, cd) += sum_h Eb(ab, h) V(h, cd)
            const double* __restrict__ Cb = Bp + S::POA;
            if constexpr (K::WREG) {
#pragma unroll
                for (int j = 0; j < K::WSLOTS; ++j) {
                    const int w = lane + TW * j;
                    if (w < S::NE * S::NF) {
                        const int ab = w / S::NF, f = w - ab * S::NF;
                        double acc = Wr[j];
                        const int c1 = tab_cbo[ab + 1];
                        for (int c = tab_cbo[ab]; c < c1; ++c) acc += __ldg(Cb + c) * V[tab_cbh[c] * S::NF + f];
                        Wr[j] = acc;
                    }
                }
            } else {
                for (int w = lane; w < S::NE * S::NF; w += TW) {
                    const int ab = w / S::NF, f = w - ab * S::NF;
                    double acc = Ws[w];
                    const int c1 = tab_cbo[ab + 1];
                    for (int c = tab_cbo[ab]; c < c1; ++c) acc += __ldg(Cb + c) * V[tab_cbh[c] * S::NF + f];
                    Ws[w] = acc;
                }
            }
            team_sync<TW, TPB>();
        }

        // ================= epilogue: transforms + scatter =================
        double* P0;
        double* P1;
        if constexpr (K::WREG) {
            P0 = ts;
            P1 = ts + S::NE * S::NF;
#pragma unroll
            for (int j = 0; j < K::WSLOTS; ++j) {
                const int w = lane + TW * j;
                if (w < S::NE * S::NF) P0[w] = Wr[j];
            }
            team_sync<TW, TPB>();
        } else {
            P0 = Ws;
            P1 = ts;
        }
        eri_epilogue<LA, LB, LC, LD, TW, TPB>(a, pb, pk, bra, ket, P0, P1, lane);
        team_sync<TW, TPB>();
    }
}

} // namespace gci
