// eri_hermite.cuh -- product-mode ERI stages in Hermite-matrix form on the
// FP64 tensor-core path (DMMA, mma.sync m8n8k4 f64).
//
// For a row shell pair AB (primitive pairs i) and a column shell pair CD
// (primitive pairs k), every (ab|cd) of the McMurchie-Davidson sum of the
// reference (auto2e_WMatrix_part1.f90:743-812, Hermite recursions of
// auto2e_Hermite.f90) is
//     (r|J) = sum_i sum_h Er_i(r, h) sum_k sum_g R_ik(h + g) Ec_k(g, J)
// where r runs over the (spherical, normalised) functions of the row pair,
// J over the requested functions of the column pair, and
//     Er_i(r, h) = K_ab c_a c_b sum_{a,b} T_A(r_a, a) T_B(r_b, b) E^{ab}_i(h)
//     Ec_k(g, J) = (-1)^|g| K_cd c_c c_d sum_{c,d} T_C(J_c, c) T_D(J_d, d) E^{cd}_k(g)
// are the pair's Hermite vectors (E^{ab} the two-centre Hermite coefficients
// of the primitive pair, T the normalisation x solid-harmonic transforms).
// The Cartesian -> spherical transforms of the reference
// (auto2e_SpherTransf.f90, auto2e_Normalize_*) are thus applied to the
// Hermite coefficients once per primitive pair instead of to every
// contracted quartet, and the ket side carries only the columns a stage
// keeps (pivot columns in the full-dimension stage, Step2.f90:242-419).
//
// Per primitive quartet the inner sum is a dense product
//     X_i(h, J) += R~_ik(h, g) Ec_k(g, J),    R~(h, g) = R(h + g)
// of H1 x H2 by H2 x nJ, and per row primitive pair O(r, J) += Er_i(r, h) X_i(h, J).
// One warp evaluates one (row pair, column chunk) task: R_ik in warp-private
// shared memory (level recursion, Helgaker 9.9.18-20), the Hankel operand
// gathered from it through a per-block index table, the column vectors read
// as ready-made B fragments, X and O in registers as DMMA accumulators; X is
// turned into B fragments of the row product by warp shuffles.
#pragma once
#include "gci_common.h"
#include "boys.cuh"
#include <type_traits>

namespace gci {

template <int L1, int L2, int NT>
struct HmShape {
    static constexpr int LT = L1 + L2;
    static constexpr int H1 = herm_n(L1), H2 = herm_n(L2), HT = herm_n(LT);
    static constexpr int MT = hm_mt(L1), KT = hm_kt(L2), MTO = hm_mto(L1);
    static constexpr int RSTR = hm_row_stride(L1), CSTR = hm_col_stride(L2, NT);
    static constexpr int KB = 32;          // column primitive pairs prepared at once (one per lane)
    static constexpr int FS = LT + 4;      // per prepared primitive pair: F_0..F_LT, X, Y, Z
    static constexpr int RS = HT + 1;      // R buffer, the last slot stays zero (padding of the gather)
    static constexpr int OS = MTO * 8 * NT * 8;   // output block O(r, J), fragment order [MTO][NT][32][2]
    static constexpr int WS = 3 * RS + KB * FS + OS;
    // eight warps share the block's tables; (f,f|f,f) with three column tiles
    // fills 226 KB of shared memory
    static constexpr int WARPS = 8, TPB = 32 * WARPS;
    // independent accumulator sets over alternating k-steps, so that at least
    // ~12 tensor-core products are in flight per warp when the tile count is small
    static constexpr int ACC0 = (12 + MT * NT - 1) / (MT * NT);
    static constexpr int ACC = ACC0 > 4 ? 4 : ACC0;
    // blocks per SM the launch bounds ask for: two when the accumulators are few
    static constexpr int MINB = ACC * MT * NT * 2 <= 24 ? 2 : 1;
    // the next k-step's Hankel fragments are loaded one step ahead (registers: 2 MT)
    static constexpr bool APF = MT <= 7;
    static constexpr size_t smem_bytes()
    {
        return sizeof(double) * ((size_t)WARPS * WS + HT) + sizeof(int) * (size_t)HT +
               sizeof(short) * (size_t)MT * KT * 32;
    }
};

template <int I, int N, class Fn>
__device__ __forceinline__ void hm_static_for(Fn&& fn)
{
    if constexpr (I < N) {
        fn(std::integral_constant<int, I>{});
        hm_static_for<I + 1, N>(fn);
    }
}

// D = A B + D for one 8x8x4 tile: lane l holds A[l/4][l%4], B[l%4][l/4] and
// D[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

// One level of the Hermite Coulomb recursion (Helgaker 9.9.18-20):
//   R^{(j)}_{tuv} = d R^{(j+1)}_{tuv - e} + (n - 1) R^{(j+1)}_{tuv - 2e}
// along the first nonzero axis e of (t,u,v), with component n and d = X, Y or
// Z, for every t+u+v <= LT - j, from `src` (level j+1) into `dst`; the
// (0,0,0) entry takes F_j.  tab_rec packs the byte offsets of the two source
// entries (bits 0-11, 12-23) and of d within fk[LT+1..LT+3] (bits 24-31).
template <int LT>
__device__ __forceinline__ void hm_level(int j, const double* __restrict__ fk, const double* src, double* dst,
                                         const int* __restrict__ tab_rec, const double* __restrict__ tab_coef,
                                         int lane)
{
    const int nent = herm_n(LT - j);
    const double Fj = fk[j];
    const char* sb = reinterpret_cast<const char*>(src);
    const char* db = reinterpret_cast<const char*>(fk + LT + 1);
    for (int h = lane; h < nent; h += 32) {
        const int rc = tab_rec[h];
        const double d = *reinterpret_cast<const double*>(db + (rc >> 24));
        const double r1 = *reinterpret_cast<const double*>(sb + (rc & 0xfff));
        const double r2 = *reinterpret_cast<const double*>(sb + ((rc >> 12) & 0xfff));
        const double r = fma(tab_coef[h], r2, d * r1);
        dst[h] = h == 0 ? Fj : r;
    }
}

template <int L1, int L2, int NT>
__global__ void __launch_bounds__(HmShape<L1, L2, NT>::TPB, HmShape<L1, L2, NT>::MINB)
k_eri_hm(const HmArgs a)
{
    using S = HmShape<L1, L2, NT>;
    constexpr int LT = S::LT, HT = S::HT, MT = S::MT, KT = S::KT, MTO = S::MTO, ACC = S::ACC;
    extern __shared__ double smem[];
    double* tab_coef = smem + (size_t)S::WARPS * S::WS;
    int* tab_rec = reinterpret_cast<int*>(tab_coef + HT);
    short* tab_gidx = reinterpret_cast<short*>(tab_rec + HT);

    for (int c = threadIdx.x; c < HT; c += S::TPB) {
        const int t = herm_t(c), u = herm_u(c), v = herm_v(c);
        int ax = 0, i1 = 0, i2 = 0, n = 0;
        if (t > 0) { ax = 0; n = t; i1 = herm_idx(t - 1, u, v); i2 = t > 1 ? herm_idx(t - 2, u, v) : 0; }
        else if (u > 0) { ax = 1; n = u; i1 = herm_idx(t, u - 1, v); i2 = u > 1 ? herm_idx(t, u - 2, v) : 0; }
        else if (v > 0) { ax = 2; n = v; i1 = herm_idx(t, u, v - 1); i2 = v > 1 ? herm_idx(t, u, v - 2) : 0; }
        tab_rec[c] = (8 * i1) | ((8 * i2) << 12) | ((8 * ax) << 24);
        tab_coef[c] = n > 1 ? (double)(n - 1) : 0.0;
    }
    // A fragment (mt, ks) of the Hankel operand: lane l reads R(h + g) with
    // h = 8 mt + l/4, g = 4 ks + l%4; padding reads the zero slot HT
    for (int c = threadIdx.x; c < MT * KT * 32; c += S::TPB) {
        const int l = c & 31, f = c >> 5;
        const int mt = f / KT, ks = f - mt * KT;
        const int h = 8 * mt + (l >> 2), g = 4 * ks + (l & 3);
        int idx = HT;
        if (h < S::H1 && g < S::H2)
            idx = herm_idx(herm_t(h) + herm_t(g), herm_u(h) + herm_u(g), herm_v(h) + herm_v(g));
        tab_gidx[c] = (short)idx;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* Rb = smem + (size_t)warp * S::WS;   // three R buffers of RS doubles
    double* Fk = Rb + 3 * S::RS;
    double* Os = Fk + S::KB * S::FS;
    if (lane < 3) Rb[lane * S::RS + HT] = 0.0;
    __syncthreads();

    const int64_t ntasks = a.nrows * a.nchunks;
    for (;;) {
        // tasks in row-major order (a row pair's chunks are consecutive), taken
        // one at a time from the launch's counter
        unsigned long long t0 = 0;
        if (lane == 0) t0 = atomicAdd(a.counter, 1ULL);
        const int64_t task = (int64_t)__shfl_sync(0xffffffffu, t0, 0);
        if (task >= ntasks) break;
        const int64_t rix = task / a.nchunks;
        const HmChunk ch = a.chunks[a.chunk_ids[task - rix * a.nchunks]];
        const int rp = a.rows[rix];
        const ShellPairDev pr = a.pairs[rp];
        const ShellPairDev pc = a.pairs[ch.pair];
        const int nb = pr.npp, nk = pc.npp;
        const int rsr = pp_record(pr.l1, pr.l2), rsc = pp_record(pc.l1, pc.l2);
        const double* __restrict__ rrec = a.pp + pr.rec_off;
        const double* __restrict__ crec = a.pp + pc.rec_off;
        const double* __restrict__ rowv = a.rowvec + a.rowvec_off[rp];
        const double* __restrict__ colv = a.colvec + ch.vec_off;
        const int first = pr.swap ? pr.s2 : pr.s1, second = pr.swap ? pr.s1 : pr.s2;
        const int n1 = __ldg(a.sh_nfunc + first);
        const int nR = n1 * __ldg(a.sh_nfunc + second);

        // each lane owns entries 2 lane + {0,1} of every 64-entry tile of the block
        for (int w = 2 * lane; w < S::OS; w += 64) { Os[w] = 0.0; Os[w + 1] = 0.0; }

        for (int i = 0; i < nb; ++i) {
            const double* __restrict__ Bp = rrec + (size_t)i * rsr;
            const double P = __ldg(Bp + 0), px = __ldg(Bp + 1), py = __ldg(Bp + 2), pz = __ldg(Bp + 3);
            double X[ACC][MT][NT][2];
#pragma unroll
            for (int u = 0; u < ACC; ++u)
#pragma unroll
                for (int m = 0; m < MT; ++m)
#pragma unroll
                    for (int n = 0; n < NT; ++n) X[u][m][n][0] = X[u][m][n][1] = 0.0;

            for (int k0 = 0; k0 < nk; k0 += S::KB) {
                const int kn = (nk - k0) < S::KB ? (nk - k0) : S::KB;
                for (int kk = lane; kk < kn; kk += 32) {
                    // Boys values scaled by 2 pi^{5/2} / (PQ sqrt(P+Q+kappa PQ)) (auto2e_WMatrix_part1.f90:134)
                    // and (-2 alpha)^m, and P - Q, of this row primitive with column primitive k0 + kk
                    const double* __restrict__ Kp = crec + (size_t)(k0 + kk) * rsc;
                    const double Q = __ldg(Kp + 0);
                    const double dx = px - __ldg(Kp + 1), dy = py - __ldg(Kp + 2), dz = pz - __ldg(Kp + 3);
                    const double PQ = P * Q;
                    const double den = P + Q + a.kappa * PQ;
                    const double alpha = PQ / den;
                    const double pref = 34.986836655249725 / (PQ * sqrt(den));
                    double F[LT + 1];
                    boys_fm<LT>(alpha * (dx * dx + dy * dy + dz * dz), a.boys, F);
                    double* fk = Fk + kk * S::FS;
                    double pw = pref;
                    const double m2a = -2.0 * alpha;
#pragma unroll
                    for (int m = 0; m <= LT; ++m) { fk[m] = F[m] * pw; pw *= m2a; }
                    fk[LT + 1] = dx; fk[LT + 2] = dy; fk[LT + 3] = dz;
                }
                __syncwarp();
                // R of the block's first primitive quartet; every later one is built
                // level by level between the tensor-core steps of its predecessor
                double* C = Rb;
                double* src = Rb + S::RS;
                double* dst = Rb + 2 * S::RS;
                if (lane == 0) src[0] = Fk[LT];
                __syncwarp();
#pragma unroll 1
                for (int j = LT - 1; j >= 0; --j) {
                    hm_level<LT>(j, Fk, src, C, tab_rec, tab_coef, lane);
                    __syncwarp();
                    double* tmp = src; src = C; C = tmp;
                }
                { double* tmp = src; src = C; C = tmp; }   // C holds R^{(0)}
                for (int kk = 0; kk < kn; ++kk) {
                    const bool more = kk + 1 < kn;
                    const double* fkn = Fk + (kk + 1) * S::FS;
                    if (more && lane == 0) src[0] = fkn[LT];
                    __syncwarp();
                    // X(h, J) += R~(h, g) Ec(g, J), with the next quartet's recursion
                    // levels spread over the k-steps
                    const double* __restrict__ cv = colv + (size_t)(k0 + kk) * S::CSTR + lane;
                    double bn[NT];
#pragma unroll
                    for (int n = 0; n < NT; ++n) bn[n] = __ldg(cv + n * 32);
                    double an[S::APF ? MT : 1];
                    if constexpr (S::APF) {
#pragma unroll
                        for (int m = 0; m < MT; ++m) an[m] = C[tab_gidx[m * KT * 32 + lane]];
                    }
                    int q = 0;
#pragma unroll 1
                    for (int ks0 = 0; ks0 < KT; ks0 += ACC) {
                        hm_static_for<0, ACC>([&](auto U) {
                            constexpr int u = decltype(U)::value;
                            const int ks = ks0 + u;
                            if (ks < KT) {
                                double b[NT];
#pragma unroll
                                for (int n = 0; n < NT; ++n) b[n] = bn[n];
                                if (ks + 1 < KT) {
#pragma unroll
                                    for (int n = 0; n < NT; ++n) bn[n] = __ldg(cv + ((ks + 1) * NT + n) * 32);
                                }
                                const short* gi = tab_gidx + ks * 32 + lane;
                                if constexpr (S::APF) {
                                    double av[MT];
#pragma unroll
                                    for (int m = 0; m < MT; ++m) av[m] = an[m];
                                    if (ks + 1 < KT) {
#pragma unroll
                                        for (int m = 0; m < MT; ++m) an[m] = C[gi[m * KT * 32 + 32]];
                                    }
#pragma unroll
                                    for (int m = 0; m < MT; ++m)
#pragma unroll
                                        for (int n = 0; n < NT; ++n) dmma884(X[u][m][n], av[m], b[n]);
                                } else {
#pragma unroll
                                    for (int m = 0; m < MT; ++m) {
                                        const double av = C[gi[m * KT * 32]];
#pragma unroll
                                        for (int n = 0; n < NT; ++n) dmma884(X[u][m][n], av, b[n]);
                                    }
                                }
                                const int qe = more ? ((ks + 1) * LT) / KT : 0;
                                for (; q < qe; ++q) {
                                    hm_level<LT>(LT - 1 - q, fkn, src, dst, tab_rec, tab_coef, lane);
                                    __syncwarp();
                                    double* tmp = src; src = dst; dst = tmp;
                                }
                            }
                        });
                    }
                    // the next quartet's R^{(0)} is in src; the free buffers rotate
                    double* tmp = C; C = src; src = tmp;
                    __syncwarp();
                }
            }
            // O(r, J) += Er_i(r, h) X(h, J); the B fragment of k-step ks (h = 4 ks + l%4,
            // J = 8 n + l/4) is held by lane 16 (ks%2) + 4 (l%4) + l/8 of X[ks/2][n]
            if constexpr (ACC > 1) {
#pragma unroll
                for (int u = 1; u < ACC; ++u)
#pragma unroll
                    for (int m = 0; m < MT; ++m)
#pragma unroll
                        for (int n = 0; n < NT; ++n) { X[0][m][n][0] += X[u][m][n][0]; X[0][m][n][1] += X[u][m][n][1]; }
            }
            const double* __restrict__ rv = rowv + (size_t)i * S::RSTR + lane;
            const int src0 = ((lane & 3) << 2) + (lane >> 3);
            const bool odd = (lane >> 2) & 1;
            // one 8-row tile of O at a time (even and odd k-steps in separate
            // accumulators), added into the warp's block in shared memory
#pragma unroll 1
            for (int m = 0; m < MTO; ++m) {
                if (8 * m >= nR) break;
                double acc[2][NT][2];
#pragma unroll
                for (int n = 0; n < NT; ++n) acc[0][n][0] = acc[0][n][1] = acc[1][n][0] = acc[1][n][1] = 0.0;
#pragma unroll
                for (int ks = 0; ks < 2 * MT; ++ks) {
                    const double av = __ldg(rv + (m * 2 * MT + ks) * 32);
                    const int srcl = src0 + ((ks & 1) << 4);
#pragma unroll
                    for (int n = 0; n < NT; ++n) {
                        const double v0 = __shfl_sync(0xffffffffu, X[0][ks >> 1][n][0], srcl);
                        const double v1 = __shfl_sync(0xffffffffu, X[0][ks >> 1][n][1], srcl);
                        dmma884(acc[ks & 1][n], av, odd ? v1 : v0);
                    }
                }
                double* o = Os + (m * NT) * 64 + 2 * lane;
#pragma unroll
                for (int n = 0; n < NT; ++n) {
                    o[n * 64] += acc[0][n][0] + acc[1][n][0];
                    o[n * 64 + 1] += acc[0][n][1] + acc[1][n][1];
                }
            }
        }

        // scatter: element (m, n, l, e) of the block is O(8 m + l/4, 8 n + 2 (l%4) + e)
#pragma unroll 1
        for (int m = 0; m < MTO; ++m) {
            const int r = 8 * m + (lane >> 2);
            if (r >= nR) continue;
#pragma unroll
            for (int n = 0; n < NT; ++n)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int J = 8 * n + 2 * (lane & 3) + e;
                    if (J >= ch.ncol) continue;
                    const int col = a.colout[ch.col_off + J];
                    if (col < 0) continue;
                    const double val = Os[(m * NT + n) * 64 + 2 * lane + e];
                    if (a.mode == kModeProduct) {
                        const int row = a.row_map[a.row_off[rp] + r];
                        if (row >= 0) a.out[row + a.ldo * (int64_t)col] = val;
                    } else {
                        const int i1 = r % n1, i2 = r / n1;
                        const int64_t p = __ldg(a.sh_loc + first) + i1, q = __ldg(a.sh_loc + second) + i2;
                        a.out[(p * a.nao + q) * a.jcount + col] = val;
                        if (first != second) a.out[(q * a.nao + p) * a.jcount + col] = val;
                    }
                }
        }
    }
}

} // namespace gci

namespace gci {

using HmLaunchFn = cudaError_t (*)(const HmArgs&, cudaStream_t);

// The shared-memory attribute is set on every launch: it belongs to the
// current device, and the library may be called on several devices.
template <int L1, int L2, int NT>
static cudaError_t launch_hm(const HmArgs& a, cudaStream_t st)
{
    using S = HmShape<L1, L2, NT>;
    const int64_t ntasks = a.nrows * a.nchunks;
    if (ntasks <= 0) return cudaSuccess;
    auto kern = k_eri_hm<L1, L2, NT>;
    const size_t smem = S::smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // persistent: as many blocks as are resident at once; warps take tasks from a.counter
    int dev = 0, nsm = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, S::TPB, smem)) != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int64_t blocks = (ntasks + S::WARPS - 1) / S::WARPS;
    const int64_t cap = (int64_t)nsm * per_sm;
    if (blocks > cap) blocks = cap;
    kern<<<(unsigned)blocks, S::TPB, smem, st>>>(a);
    return cudaGetLastError();
}

// tab[L1][L2][NT - 1] for L2 = 0 .. kMaxPairL and NT = 1 .. hm_max_nt(L1)
template <int L1, int L2, int NT = 1>
static void register_hm_nt(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT])
{
    tab[L1][L2][NT - 1] = &launch_hm<L1, L2, NT>;
    if constexpr (NT < hm_max_nt(L1)) register_hm_nt<L1, L2, NT + 1>(tab);
}

template <int L1, int L2 = 0>
static void register_hm_row(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT])
{
    register_hm_nt<L1, L2>(tab);
    if constexpr (L2 < kMaxPairL) register_hm_row<L1, L2 + 1>(tab);
}

void register_hm_0(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]);
void register_hm_1(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]);
void register_hm_2(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]);
void register_hm_3(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]);
void register_hm_4(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]);
void register_hm_5(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]);
void register_hm_6(HmLaunchFn (*tab)[kMaxPairL + 1][kHmMaxNT]);

} // namespace gci
