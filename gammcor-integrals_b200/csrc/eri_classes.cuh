// eri_classes.cuh -- launcher template of the class kernels; each
// eri_classes_*.cu translation unit instantiates a share of the 55 canonical
// classes so that they compile in parallel.
#pragma once
#include "eri_engine.cuh"
#include "eri_ketfirst.cuh"

namespace gci {

using LaunchFn = void (*)(const EriArgs&, cudaStream_t);

constexpr int type_lhi(int t) { return t >= 6 ? 3 : (t >= 3 ? 2 : (t >= 1 ? 1 : 0)); }
constexpr int type_llo(int t) { return t - pair_type(type_lhi(t), 0); }

// Grid: the task list with a cap of 64 blocks per SM (grid-stride loop inside).
template <int TB, int TK>
static void launch_class(const EriArgs& args, cudaStream_t st)
{
    constexpr int LA = type_lhi(TB), LB = type_llo(TB), LC = type_lhi(TK), LD = type_llo(TK);
    using G = EriTeam<LA, LB, LC, LD>;
    const size_t smem = G::smem_bytes();
    auto kern = k_eri_class<LA, LB, LC, LD>;
    // the attribute belongs to the current device: set it on every launch, so that
    // launches on any device the library is called on see it
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int64_t ntasks = (args.mode == kModeDiagonal) ? args.nbra : args.nbra * args.nket;
    if (ntasks <= 0) return;
    int64_t blocks = (ntasks + G::NT - 1) / G::NT;
    const int64_t cap = 148LL * 64;
    if (blocks > cap) blocks = cap;
    kern<<<(unsigned)blocks, G::TPB, smem, st>>>(args);
}

// Ket-first kernel (eri_ketfirst.cuh), built for bra types from (d,s) up in
// three team widths (32, 64, 128 lanes per quartet); grid capped at 64 blocks
// per SM with a grid-stride loop inside.
constexpr int kNumKfWidths = 3;
constexpr int kf_width(int w) { return w == 0 ? 32 : (w == 1 ? 64 : 128); }

template <int TB, int TK, int TWQ>
static void launch_kf(const EriArgs& args, cudaStream_t st)
{
    constexpr int LA = type_lhi(TB), LB = type_llo(TB), LC = type_lhi(TK), LD = type_llo(TK);
    using K = KfShape<LA, LB, LC, LD, TWQ>;
    const size_t smem = K::smem_bytes();
    auto kern = k_eri_kf<LA, LB, LC, LD, TWQ>;
    // the attribute belongs to the current device: set it on every launch, so that
    // launches on any device the library is called on see it
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int64_t ntasks = (args.mode == kModeDiagonal) ? args.nbra : args.nbra * args.nket;
    if (ntasks <= 0) return;
    int64_t blocks = (ntasks + K::TEAMS - 1) / K::TEAMS;
    const int64_t cap = 148LL * 64;
    if (blocks > cap) blocks = cap;
    kern<<<(unsigned)blocks, K::TPB, smem, st>>>(args);
}

// which widths are built: a warp only while a quartet's W block stays small,
// 64 lanes up to 4096 elements, 128 lanes only from 512 elements; all within 227 KB
template <int TB, int TK, int W>
constexpr bool has_kf()
{
    if (TB < 3 || TK > TB) return false;
    constexpr int LA = type_lhi(TB), LB = type_llo(TB), LC = type_lhi(TK), LD = type_llo(TK);
    constexpr int nw = ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD);
    if (W == 0 && nw > 4096) return false;
    if (W == 1 && nw > 6000) return false;
    if (W == 2 && nw < 512) return false;
    return KfShape<LA, LB, LC, LD, kf_width(W)>::smem_bytes() <= 227 * 1024;
}

template <int TB, int W, int TK = TB>
static void register_row_kf(LaunchFn (*tab)[kNumPairTypes][kNumPairTypes])
{
    if constexpr (has_kf<TB, TK, W>()) tab[W][TB][TK] = &launch_kf<TB, TK, kf_width(W)>;
    if constexpr (TK > 0) register_row_kf<TB, W, TK - 1>(tab);
}

template <int TB>
static void register_row_kf_all(LaunchFn (*tab)[kNumPairTypes][kNumPairTypes])
{
    register_row_kf<TB, 0>(tab);
    register_row_kf<TB, 1>(tab);
    register_row_kf<TB, 2>(tab);
}

// register the classes (TB, TK) for TK = 0..TB into a launch table
template <int TB, int TK = TB>
static void register_row(LaunchFn (*tab)[kNumPairTypes])
{
    tab[TB][TK] = &launch_class<TB, TK>;
    if constexpr (TK > 0) register_row<TB, TK - 1>(tab);
}

void register_eri_classes_a(LaunchFn (*tab)[kNumPairTypes]);
void register_eri_kf_a(LaunchFn (*tab)[kNumPairTypes][kNumPairTypes]);
void register_eri_kf_b(LaunchFn (*tab)[kNumPairTypes][kNumPairTypes]);
void register_eri_kf_c(LaunchFn (*tab)[kNumPairTypes][kNumPairTypes]);
void register_eri_kf_d(LaunchFn (*tab)[kNumPairTypes][kNumPairTypes]);

} // namespace gci
