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
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set = true;
    }
    const int64_t ntasks = (args.mode == kModeDiagonal) ? args.nbra : args.nbra * args.nket;
    if (ntasks <= 0) return;
    int64_t blocks = (ntasks + G::NT - 1) / G::NT;
    const int64_t cap = 148LL * 64;
    if (blocks > cap) blocks = cap;
    kern<<<(unsigned)blocks, G::TPB, smem, st>>>(args);
}

// Ket-first kernel (eri_ketfirst.cuh), built for bra types from (d,s) up:
// a warp or a 128-thread block per quartet, grid capped at 64 blocks per SM
// with a grid-stride loop inside.
template <int TB, int TK>
static void launch_kf(const EriArgs& args, cudaStream_t st)
{
    constexpr int LA = type_lhi(TB), LB = type_llo(TB), LC = type_lhi(TK), LD = type_llo(TK);
    using K = KfShape<LA, LB, LC, LD>;
    const size_t smem = K::smem_bytes();
    auto kern = k_eri_kf<LA, LB, LC, LD>;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_set = true;
    }
    const int64_t ntasks = (args.mode == kModeDiagonal) ? args.nbra : args.nbra * args.nket;
    if (ntasks <= 0) return;
    int64_t blocks = (ntasks + K::TEAMS - 1) / K::TEAMS;
    const int64_t cap = 148LL * 64;
    if (blocks > cap) blocks = cap;
    kern<<<(unsigned)blocks, K::TPB, smem, st>>>(args);
}

constexpr bool has_kf(int tb, int tk) { return tb >= 3 && tk <= tb; }

template <int TB, int TK = TB>
static void register_row_kf(LaunchFn (*tab)[kNumPairTypes])
{
    if constexpr (has_kf(TB, TK)) tab[TB][TK] = &launch_kf<TB, TK>;
    if constexpr (TK > 0) register_row_kf<TB, TK - 1>(tab);
}

// register the classes (TB, TK) for TK = 0..TB into a launch table
template <int TB, int TK = TB>
static void register_row(LaunchFn (*tab)[kNumPairTypes])
{
    tab[TB][TK] = &launch_class<TB, TK>;
    if constexpr (TK > 0) register_row<TB, TK - 1>(tab);
}

void register_eri_classes_a(LaunchFn (*tab)[kNumPairTypes]);
void register_eri_classes_b(LaunchFn (*tab)[kNumPairTypes]);
void register_eri_classes_c(LaunchFn (*tab)[kNumPairTypes]);
void register_eri_classes_d(LaunchFn (*tab)[kNumPairTypes]);
void register_eri_kf_a(LaunchFn (*tab)[kNumPairTypes]);
void register_eri_kf_b(LaunchFn (*tab)[kNumPairTypes]);
void register_eri_kf_c(LaunchFn (*tab)[kNumPairTypes]);
void register_eri_kf_d(LaunchFn (*tab)[kNumPairTypes]);

} // namespace gci
