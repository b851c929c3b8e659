// gci_common.h -- definitions shared by the host runtime and the sm_100a kernels
// of the integral-direct Cholesky ERI library.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define GCI_HD __host__ __device__ __forceinline__

namespace gci {

// Highest angular momentum handled by the GPU ERI kernels (f shells).  The
// reference engine goes to h (auto2e.f90:275); classes above f are rejected
// with an error by the host runtime.
constexpr int kMaxL = 3;
constexpr int kMaxPairL = 2 * kMaxL;          // bra or ket level
constexpr int kMaxLT = 2 * kMaxPairL;         // total Hermite level
constexpr int kMaxDerivLT = kMaxLT + 1;       // adjoint kernels shift one level up
constexpr int kBoysMaxM = 20;                 // table order, 4*AUTO2E_MAXL (Cholesky_Gammcor.f90:350)
constexpr int kBoysNInt = 500;                // intervals on [0, 25)  (boys.f90:20-21,43)
constexpr double kBoysXAsym = 25.0;
constexpr double kBoysDelta = kBoysXAsym / kBoysNInt;
constexpr double kPi = 3.14159265358979323846264338327950288;

GCI_HD constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
GCI_HD constexpr int cart_off(int l) { return l * (l + 1) * (l + 2) / 6; }
GCI_HD constexpr int herm_n(int n) { return (n + 1) * (n + 2) * (n + 3) / 6; }
GCI_HD constexpr int tri(int l) { return (l + 1) * (l + 2) / 2; }
// Hermite index, level-major: all (t,u,v) with t+u+v < n precede level n.
GCI_HD constexpr int herm_idx(int t, int u, int v)
{
    return (t + u + v) * (t + u + v + 1) * (t + u + v + 2) / 6 + (u + v) * (u + v + 1) / 2 + v;
}
// Position of (lx,ly,lz) within its level, Auto2e order (lx desc, ly desc).
GCI_HD constexpr int cart_pos(int ly, int lz) { return (ly + lz) * (ly + lz + 1) / 2 + lz; }
// Shell pair type for l_hi >= l_lo: 0..9 for l <= 3.
GCI_HD constexpr int pair_type(int lhi, int llo) { return lhi * (lhi + 1) / 2 + llo; }
constexpr int kNumPairTypes = pair_type(kMaxL, kMaxL) + 1;
// Hermite level l_hi + l_lo of pair type t.
GCI_HD constexpr int type_lsum(int t)
{
    int hi = 0;
    while (pair_type(hi + 1, 0) <= t) ++hi;
    return hi + (t - pair_type(hi, 0));
}

// Two-centre Hermite coefficients E^{ij}_t of (x-A)^i (x-B)^j exp(-p (x-P)^2),
// i <= la, j <= lb, t <= i+j, one table per axis: block (i, j) starts at
// e2_off(la, i, j) (j major, then i), e2_size entries in all.
GCI_HD constexpr int e2_off(int la, int i, int j)
{
    return (la + 1) * j * (j + 1) / 2 + j * la * (la + 1) / 2 + i * (j + 1) + i * (i - 1) / 2;
}
GCI_HD constexpr int e2_size(int la, int lb) { return (la + 1) * (lb + 1) * (la + lb + 2) / 2; }

// ------------------------------------------------------------ index helpers (compile time and device)
GCI_HD constexpr int cart_level(int g) { int l = 0; while (cart_off(l + 1) <= g) ++l; return l; }
GCI_HD constexpr int cart_x(int g) { int l = cart_level(g), p = g - cart_off(l), s = 0; while ((s + 1) * (s + 2) / 2 <= p) ++s; return l - s; }
GCI_HD constexpr int cart_z(int g) { int l = cart_level(g), p = g - cart_off(l), s = 0; while ((s + 1) * (s + 2) / 2 <= p) ++s; return p - s * (s + 1) / 2; }
GCI_HD constexpr int cart_y(int g) { return cart_level(g) - cart_x(g) - cart_z(g); }
GCI_HD constexpr int herm_level(int h) { int n = 0; while (herm_n(n) <= h) ++n; return n; }
GCI_HD constexpr int herm_v(int h) { int n = herm_level(h), p = h - (n > 0 ? herm_n(n - 1) : 0), s = 0; while ((s + 1) * (s + 2) / 2 <= p) ++s; return p - s * (s + 1) / 2; }
GCI_HD constexpr int herm_u(int h) { int n = herm_level(h), p = h - (n > 0 ? herm_n(n - 1) : 0), s = 0; while ((s + 1) * (s + 2) / 2 <= p) ++s; return s - (p - s * (s + 1) / 2); }
GCI_HD constexpr int herm_t(int h) { return herm_level(h) - herm_u(h) - herm_v(h); }
GCI_HD constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Cartesian pair e = (a, b) of shells (la, lb), b fastest: its Hermite extent
// along each axis and the offset of its coefficient block in a per-axis table.
GCI_HD constexpr int pair_ga(int la, int lb, int e) { return cart_off(la) + e / ncart(lb); }
GCI_HD constexpr int pair_gb(int la, int lb, int e) { return cart_off(lb) + e % ncart(lb); }
GCI_HD constexpr int pair_x(int la, int lb, int e) { return cart_x(pair_ga(la, lb, e)) + cart_x(pair_gb(la, lb, e)); }
GCI_HD constexpr int pair_y(int la, int lb, int e) { return cart_y(pair_ga(la, lb, e)) + cart_y(pair_gb(la, lb, e)); }
GCI_HD constexpr int pair_z(int la, int lb, int e) { return cart_z(pair_ga(la, lb, e)) + cart_z(pair_gb(la, lb, e)); }
GCI_HD constexpr int pair_ox(int la, int lb, int e) { return e2_off(la, cart_x(pair_ga(la, lb, e)), cart_x(pair_gb(la, lb, e))); }
GCI_HD constexpr int pair_oy(int la, int lb, int e) { return e2_off(la, cart_y(pair_ga(la, lb, e)), cart_y(pair_gb(la, lb, e))); }
GCI_HD constexpr int pair_oz(int la, int lb, int e) { return e2_off(la, cart_z(pair_ga(la, lb, e)), cart_z(pair_gb(la, lb, e))); }
GCI_HD constexpr int pair_supp(int la, int lb, int e)
{
    return (pair_x(la, lb, e) + 1) * (pair_y(la, lb, e) + 1) * (pair_z(la, lb, e) + 1);
}

// Number of Hermite products E^{ab}_{tuv} = E^x E^y E^z over all Cartesian pairs
// of shells (la, lb): the product table of a primitive-pair record.
GCI_HD constexpr int pair_ncb(int la, int lb)
{
    int n = 0;
    for (int e = 0; e < ncart(la) * ncart(lb); ++e) n += pair_supp(la, lb, e);
    return n;
}

// Primitive-pair record of a pair (l1, l2), in doubles:
//   [0] P  [1..3] Rp  [4] K_ab c_a c_b  [5..7] Rp - A
//   [8 ..]            E^{ij}_t tables for x, y, z (e2_size each)
//   [8 + 3 e2_size ..] products E^{ab}_{tuv} for every Cartesian pair ab
//                      (b fastest), each over v outer, u, t inner
GCI_HD constexpr int pp_prod_off(int l1, int l2) { return 8 + 3 * e2_size(l1, l2); }
GCI_HD constexpr int pp_record(int l1, int l2) { return pp_prod_off(l1, l2) + pair_ncb(l1, l2); }

// Output modes of the ERI kernels.
enum EriMode : int {
    kModeProduct = 0,    // every (bra, ket) combination, written through row/col maps
    kModeDiagonal = 1,   // bra == ket, only (ab|ab) kept: out[rowmap(ab)]
    kModeDense = 2,      // bra pair x ket pair into a dense AO-pair layout (both triangles)
};

struct ShellPairDev {
    int s1, s2;          // canonical shells: s1 has the higher (or equal) L
    int swap;            // 1 if s1 is the second shell of the stored pair (A >= B index order)
    int nprim1, nprim2;
    int l1, l2;          // angular momenta of s1, s2
    int npp;             // primitive pairs kept after screening (records stored)
    int64_t rec_off;     // offset (doubles) of the first primitive-pair record
    int64_t list_off;    // offset of the kept (ga | gb << 8) list
};

struct EriArgs {
    // basis
    const double* sh_xyz;     // 3 per shell
    const int* sh_toff;       // offset of the shell's transform in tmat
    const double* tmat;       // per shell nfunc x ncart, row-major
    const int* sh_nfunc;
    const int* sh_loc;        // first AO index of each shell (dense mode)
    // pairs
    const ShellPairDev* pairs;
    const double* pp;         // primitive-pair records
    // task space: bra list x ket list (actual orientation)
    const int* bra_ids;
    const int* ket_ids;
    int64_t nbra, nket;
    int swap_bk;              // 1: the canonical bra is the actual ket pair
    int mode;
    // output
    double* out;
    int64_t ldo;
    const int64_t* row_off;   // per pair id: offset into row_map (entries Na*Nb)
    const int* row_map;
    const int64_t* col_off;
    const int* col_map;
    int64_t nao;              // dense mode: AO count; out is [p][q][j] with j fastest
    int64_t jcount;           // dense mode: extent of the fastest index
    double kappa;
    const double* boys;       // (kBoysMaxM+1) x kBoysNInt x 5
    int* err;                 // device error word
};

// ------------------------------------------------------------ Hermite-matrix ERI path (eri_hermite.cuh)
// Largest number of spherical functions of a shell pair of Hermite level L
// (la + lb = L, la >= lb, la <= kMaxL).
GCI_HD constexpr int hm_max_nf(int L)
{
    int m = 0;
    for (int la = 0; la <= kMaxL; ++la) {
        const int lb = L - la;
        if (lb < 0 || lb > la) continue;
        const int n = (2 * la + 1) * (2 * lb + 1);
        if (n > m) m = n;
    }
    return m;
}
GCI_HD constexpr int hm_mt(int L) { return (herm_n(L) + 7) / 8; }    // 8-row tiles over a Hermite index
GCI_HD constexpr int hm_kt(int L) { return (herm_n(L) + 3) / 4; }    // 4-wide k-steps over a Hermite index
GCI_HD constexpr int hm_mto(int L) { return (hm_max_nf(L) + 7) / 8; } // 8-row tiles over the row functions
// doubles of one row primitive pair's vectors: [MTO][2 MT][32] (A fragments of the row product)
GCI_HD constexpr int hm_row_stride(int L) { return hm_mto(L) * 2 * hm_mt(L) * 32; }
// doubles of one column primitive pair's vectors in a chunk of NT column tiles: [KT][NT][32]
GCI_HD constexpr int hm_col_stride(int L, int nt) { return hm_kt(L) * nt * 32; }
constexpr int kHmMaxNT = 7;   // column tiles per task, at most (56 columns)
// Column tiles per task for rows of Hermite level L1: the 8x8 accumulator tiles of
// X (ceil(H1/8) x NT) stay at about 30 or fewer (two doubles per lane each).
GCI_HD constexpr int hm_max_nt(int L1) { return L1 <= 3 ? 7 : (L1 == 4 ? 5 : (L1 == 5 ? 4 : 3)); }

// A group of at most 8 * NT requested columns of one column pair.
struct HmChunk {
    int pair;          // pair id (all-pair index)
    int ncol;          // columns in the chunk
    int nt;            // column tiles of its vectors (ncol <= 8 nt)
    int64_t vec_off;   // offset (doubles) of the chunk's vectors in colvec: [k][KT][NT][32]
    int64_t col_off;   // offset of the chunk's entries in colfun / colout
};

struct HmArgs {
    const ShellPairDev* pairs;
    const double* pp;            // primitive-pair records (P and the product centre at [0..3])
    const double* rowvec;        // row vectors, per pair: [i][MTO][2 MT][32]
    const int64_t* rowvec_off;   // per pair id
    const HmChunk* chunks;
    const double* colvec;
    const int* colout;           // per chunk column: output column (product) or j index (dense)
    const int* rows;             // row pair ids
    int64_t nrows;
    const int* chunk_ids;        // chunk indices of this launch
    int64_t nchunks;
    int mode;                    // kModeProduct or kModeDense
    double* out;
    int64_t ldo;
    const int64_t* row_off;      // product mode: row map of each row pair (stored-orientation functions)
    const int* row_map;
    const int* sh_nfunc;
    const int* sh_loc;
    int64_t nao, jcount;
    double kappa;
    const double* boys;
    unsigned long long* counter;   // task counter of the launch, zero at launch
};

// ------------------------------------------------------------ adjoint (Coulomb gradient) path
// Hermite level L of a shell pair (lA + lB) runs to 2 kMaxL; the derivative
// vectors reach L + 1.
constexpr int kGradMaxL = kMaxPairL;
constexpr int kGradVec = 7;   // h, gA (x,y,z), gB (x,y,z)
GCI_HD constexpr int grad_hb(int L) { return herm_n(L + 1); }   // entries of a bra vector / potential

struct GradPotArgs {
    const double* mP;        // per primitive pair: exponent sum P
    const double* mX;        // product centre
    const double* mY;
    const double* mZ;
    int64_t bra_beg, nbra;   // bra primitive pairs of level L1: global indices bra_beg ..
    int64_t ket_beg, nket;   // ket primitive pairs of level L2
    const double* hk;        // ket vectors of level L2, transposed: hk[tau * nket + k], sign (-1)^|tau| applied
    double* V;               // potentials of level L1: V[i * grad_hb(L1) + t], accumulated atomically
    int64_t chunk;           // ket primitive pairs per warp
    int64_t nchunk;          // chunks per bra primitive pair
    double kappa;
    const double* boys;
};

} // namespace gci
