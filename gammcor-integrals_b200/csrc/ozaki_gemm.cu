// ozaki_gemm.cu -- split-precision FP64 GEMM on the int8 tensor cores (tcgen05):
//     C(m x n) = alpha A(m x k) B(n x k)^T + beta C
//
// Error-free splitting (Ozaki scheme): every row r of an operand is scaled by
// 2^-E_r (E_r: the exponent of the row's largest element) and written as
// seven signed 8-bit slices, x = 2^E_r sum_{s=1..7} q_s 2^-7s + O(2^(E_r-49)).
// The products of slice pairs (s, t) are exact in int32; pairs of equal
// s + t = d share one scale 2^-7d and are summed in one TMEM accumulator
// (d = 2..9: 34 pairs, 8 accumulators of 64 int32 columns = the 512 TMEM
// columns of an SM).  The epilogue converts the eight accumulators to FP64 and
// recombines them with the row scales.  The dropped pairs (d >= 10) bound the
// error by ~k 2^-64 127^2 relative to max|A_r| max|B_c| (~1e-12 for k = 16k),
// the slices' own truncation by k 2^-48 of the same scale.
//
// Kernels:
//  * k_oz_rowexp: E_r of every row (one thread per row);
//  * k_oz_split: the seven slices of a block of rows, written in the tiled
//    image the GEMM copies into shared memory unchanged (no swizzle, K-major
//    canonical layout of 8-row x 16-byte core matrices);
//  * k_oz_gemm: one 128 x 64 output tile per CTA, K in blocks of 64 through a
//    two-stage shared-memory ring: one thread issues the 14 bulk copies
//    (cp.async.bulk, mbarrier completion) of the next block's A and B slice
//    tiles while the tensor core runs the 68 tcgen05.mma.kind::i8 (M=128,
//    N=64, K=32) of the current block into the eight TMEM accumulators, each
//    block's products committed to the mbarrier that frees its stage; the
//    epilogue reads TMEM with tcgen05.ld and writes FP64.  Every wait is
//    bounded: on expiry the CTA records GCI error 1, waits (bounded) for its
//    own copies and products, frees its TMEM and returns.
#include "gci_runtime.h"
#include <cstdint>

namespace gci {

constexpr int kOzSlices = 7;
constexpr int kOzDMax = 9;                       // pairs with s + t <= 9
constexpr int kOzBM = 128, kOzBN = 64, kOzBK = 64;
constexpr int kOzTileA = kOzBM * kOzBK;          // bytes of one A slice tile
constexpr int kOzTileB = kOzBN * kOzBK;
constexpr int kOzStage = kOzSlices * (kOzTileA + kOzTileB);   // 84 KB: all slices of one K block
constexpr int kOzStages = 2;
constexpr int kOzSmem = kOzStages * kOzStage + 128;
constexpr long long kOzSpin = 1LL << 28;         // bounded waits (~seconds)

// ------------------------------------------------------------------ row exponents
// E_r = exponent of max_l |X(r, l)| (frexp convention: |x| < 2^E); 0 for a zero row.
__global__ void k_oz_rowexp(const double* __restrict__ X, int64_t rs, int64_t ls, int64_t rows, int64_t k,
                            int* __restrict__ E)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
        double mx = 0.0;
        for (int64_t l = 0; l < k; ++l) mx = fmax(mx, fabs(X[r * rs + l * ls]));
        int e = 0;
        if (mx > 0.0) frexp(mx, &e);
        E[r] = e;
    }
}

// ------------------------------------------------------------------ slices
// Tile (s, rb, kb) of R rows x kOzBK (64) K bytes at ((s * nrb + rb) * nkb + kb) * R * 128;
// inside a tile, byte (row, kk) at ((kk / 16) * (R / 8) + row / 8) * 128 + (row % 8) * 16 + kk % 16.
template <int R>
__global__ void k_oz_split(const double* __restrict__ X, int64_t rs, int64_t ls, int64_t rows, int64_t k,
                           const int* __restrict__ E, int64_t nrb, int64_t nkb, int8_t* __restrict__ out)
{
    const int64_t nel = nrb * R * nkb * kOzBK;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
        // element order: row fastest, so that neighbouring threads read neighbouring rows
        const int64_t r = e % (nrb * R);
        const int64_t l = e / (nrb * R);
        double x = 0.0;
        if (r < rows && l < k) x = ldexp(X[r * rs + l * ls], -E[r]);
        const int64_t rb = r / R, kb = l / kOzBK;
        const int row = (int)(r % R), kk = (int)(l % kOzBK);
        const int64_t in_tile = (int64_t)((kk / 16) * (R / 8) + row / 8) * 128 + (row % 8) * 16 + kk % 16;
        const int64_t tile_stride = (int64_t)nrb * nkb * R * kOzBK;
        int8_t* o = out + (rb * nkb + kb) * (int64_t)R * kOzBK + in_tile;
#pragma unroll
        for (int s = 0; s < kOzSlices; ++s) {
            x *= 128.0;
            const double q = trunc(x);
            x -= q;
            o[s * tile_stride] = (int8_t)q;
        }
    }
}

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// true when the phase with parity `phase` has completed, false after kOzSpin polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase)
{
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < kOzSpin; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_copy(void* dst_smem, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst_smem)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// shared-memory matrix descriptor: K-major, no swizzle; LBO = byte distance of the two
// 16-byte K chunks of one K=32 step, SBO = byte distance of neighbouring 8-row groups
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3fff);
    d |= (uint64_t)((lbo >> 4) & 0x3fff) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3fff) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version (sm_100)
    return d;                 // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor of kind::i8: signed A and B, int32 D, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc_i8(int M, int N)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// ------------------------------------------------------------------ GEMM
struct OzArgs {
    const int8_t* a;       // A slice tiles (nrb_a row blocks of 128)
    const int8_t* b;       // B slice tiles (nrb_b row blocks of 64)
    const int* ea;         // row exponents of A (m) and B (n)
    const int* eb;
    int64_t m, n, nkb;     // nkb: K blocks of kOzBK
    int64_t nrb_a, nrb_b;
    double alpha, beta;
    double* c;
    int64_t ldc;
    int* err;
};

__global__ void __launch_bounds__(128, 1) k_oz_gemm(const OzArgs p)
{
    extern __shared__ __align__(1024) unsigned char oz_smem[];
    uint64_t* bar_full = reinterpret_cast<uint64_t*>(oz_smem + kOzStages * kOzStage);   // per stage: copies landed
    uint64_t* bar_empty = bar_full + kOzStages;                                         // per stage: products done
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar_empty + kOzStages);
    int* state = reinterpret_cast<int*>(tmem_slot + 1);   // ok, last committed block, last loaded block
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t cb = blockIdx.x, rb = blockIdx.y;

    if (threadIdx.x == 0) {
        for (int st = 0; st < kOzStages; ++st) {
            mbar_init(bar_full + st, 1);
            mbar_init(bar_empty + st, 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const int64_t tsa = p.nrb_a * p.nkb * (int64_t)kOzTileA;   // stride between slices of A
    const int64_t tsb = p.nrb_b * p.nkb * (int64_t)kOzTileB;
    constexpr uint32_t idesc = umma_idesc_i8(kOzBM, kOzBN);
    if (threadIdx.x == 0) {
        // block kb lives in stage kb % 2; its copies complete phase (kb / 2) % 2 of
        // bar_full[stage], its products phase (kb / 2) % 2 of bar_empty[stage]
        auto load = [&](int64_t kb) {
            const int st = (int)(kb & 1);
            int8_t* sa = reinterpret_cast<int8_t*>(oz_smem + st * kOzStage);
            int8_t* sb = sa + kOzSlices * kOzTileA;
            mbar_expect_tx(bar_full + st, kOzStage);
            for (int s = 0; s < kOzSlices; ++s) {
                bulk_copy(sa + s * kOzTileA, p.a + s * tsa + (rb * p.nkb + kb) * kOzTileA, kOzTileA, bar_full + st);
                bulk_copy(sb + s * kOzTileB, p.b + s * tsb + (cb * p.nkb + kb) * kOzTileB, kOzTileB, bar_full + st);
            }
        };
        bool ok = true;
        int64_t last_commit = -1, last_load = 0;
        load(0);
        for (int64_t kb = 0; kb < p.nkb; ++kb) {
            const int st = (int)(kb & 1);
            if (kb + 1 < p.nkb) {
                // the other stage is free once the products of block kb - 1 are done
                if (kb >= 1 && !(ok = mbar_wait(bar_empty + (st ^ 1), (uint32_t)(((kb - 1) >> 1) & 1)))) break;
                load(kb + 1);
                last_load = kb + 1;
            }
            if (!(ok = mbar_wait(bar_full + st, (uint32_t)((kb >> 1) & 1)))) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int8_t* sa = reinterpret_cast<const int8_t*>(oz_smem + st * kOzStage);
            const int8_t* sb = sa + kOzSlices * kOzTileA;
            for (int d = 2; d <= kOzDMax; ++d) {
                const uint32_t td = tmem + (uint32_t)((d - 2) * kOzBN);
                bool first = kb == 0;
                for (int s = 1; s <= kOzSlices; ++s) {
                    const int t = d - s;
                    if (t < 1 || t > kOzSlices) continue;
                    const uint32_t a0 = smem_u32(sa + (s - 1) * kOzTileA);
                    const uint32_t b0 = smem_u32(sb + (t - 1) * kOzTileB);
                    for (int kk = 0; kk < kOzBK / 32; ++kk) {
                        // K step kk covers 16-byte chunks 2kk and 2kk+1
                        const uint64_t da = umma_desc(a0 + kk * 2 * (kOzBM / 8) * 128, (kOzBM / 8) * 128, 128);
                        const uint64_t db = umma_desc(b0 + kk * 2 * (kOzBN / 8) * 128, (kOzBN / 8) * 128, 128);
                        umma_i8(td, da, db, idesc, first ? 0u : 1u);
                        first = false;
                    }
                }
            }
            umma_commit(bar_empty + st);
            last_commit = kb;
        }
        state[0] = ok ? 1 : 0;
        state[1] = (int)last_commit;
        state[2] = (int)last_load;
    }
    __syncthreads();
    bool ok = state[0] != 0;
    const int64_t last_commit = state[1], last_load = state[2];
    if (ok) ok = mbar_wait(bar_empty + (last_commit & 1), (uint32_t)((last_commit >> 1) & 1));
    ok = __syncthreads_and(ok);
    if (!ok) {
        if (threadIdx.x == 0) {
            atomicCAS(p.err, 0, 1);
            // let copies and products already issued finish (bounded) before the TMEM goes
            // (both stages: a block whose copies already landed passes at once)
            for (int64_t kb = last_load - 1; kb <= last_load; ++kb)
                if (kb >= 0) mbar_wait(bar_full + (kb & 1), (uint32_t)((kb >> 1) & 1));
            if (last_commit >= 0) mbar_wait(bar_empty + (last_commit & 1), (uint32_t)((last_commit >> 1) & 1));
        }
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // epilogue: thread (warp w, lane l) owns row 32 w + l of the tile
        const int64_t row = rb * kOzBM + warp * 32 + lane;
        double acc[kOzBN];
#pragma unroll
        for (int j = 0; j < kOzBN; ++j) acc[j] = 0.0;
#pragma unroll 1
        for (int d = kOzDMax; d >= 2; --d) {
            const double sc = ldexp(1.0, -7 * d);
#pragma unroll
            for (int c0 = 0; c0 < kOzBN; c0 += 16) {
                uint32_t v[16];
                const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((d - 2) * kOzBN + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15])
                    : "r"(addr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[c0 + j] += sc * (double)(int32_t)v[j];
            }
        }
        if (row < p.m) {
            const int er = p.ea[row];
#pragma unroll
            for (int j = 0; j < kOzBN; ++j) {
                const int64_t col = cb * kOzBN + j;
                if (col < p.n) {
                    double* cp = p.c + row + p.ldc * col;
                    const double v = p.alpha * ldexp(acc[j], er + p.eb[col]);
                    *cp = p.beta == 0.0 ? v : fma(p.beta, *cp, v);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
}

// ------------------------------------------------------------------ host side
size_t ozaki_workspace_bytes(int64_t m, int64_t n, int64_t k)
{
    const int64_t nkb = (k + kOzBK - 1) / kOzBK;
    const int64_t ma = (m + kOzBM - 1) / kOzBM * kOzBM, nb = (n + kOzBN - 1) / kOzBN * kOzBN;
    return (size_t)kOzSlices * (ma + nb) * nkb * kOzBK + sizeof(int) * (size_t)(ma + nb) + 1024;
}

int64_t ozaki_max_k() { return 18000; }

cudaError_t ozaki_dgemm_nt(int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t ars, int64_t als,
                           const double* B, int64_t brs, int64_t bls, double beta, double* C, int64_t ldc,
                           void* work, int* err, cudaStream_t st)
{
    if (m <= 0 || n <= 0) return cudaSuccess;
    if (k > ozaki_max_k()) return cudaErrorInvalidValue;   // int32 accumulators: the caller splits K
    const int64_t nkb = (k + kOzBK - 1) / kOzBK;
    const int64_t nrb_a = (m + kOzBM - 1) / kOzBM, nrb_b = (n + kOzBN - 1) / kOzBN;
    unsigned char* w = static_cast<unsigned char*>(work);
    int8_t* sa = reinterpret_cast<int8_t*>(w);
    int8_t* sb = sa + (size_t)kOzSlices * nrb_a * kOzBM * nkb * kOzBK;
    int* ea = reinterpret_cast<int*>(sb + (size_t)kOzSlices * nrb_b * kOzBN * nkb * kOzBK);
    int* eb = ea + nrb_a * kOzBM;
    const int64_t kk = k > 0 ? k : 0;
    k_oz_rowexp<<<(unsigned)std::min<int64_t>((m + 255) / 256, 148 * 8), 256, 0, st>>>(A, ars, als, m, kk, ea);
    k_oz_rowexp<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 8), 256, 0, st>>>(B, brs, bls, n, kk, eb);
    count_launch(2);
    if (k <= 0) {
        // no products: C = beta C through the epilogue of an all-zero K block
        return cudaErrorInvalidValue;
    }
    const int64_t nel_a = nrb_a * kOzBM * nkb * kOzBK, nel_b = nrb_b * kOzBN * nkb * kOzBK;
    k_oz_split<kOzBM><<<(unsigned)std::min<int64_t>((nel_a + 255) / 256, 148 * 64), 256, 0, st>>>(
        A, ars, als, m, k, ea, nrb_a, nkb, sa);
    k_oz_split<kOzBN><<<(unsigned)std::min<int64_t>((nel_b + 255) / 256, 148 * 64), 256, 0, st>>>(
        B, brs, bls, n, k, eb, nrb_b, nkb, sb);
    count_launch(2);
    cudaError_t e = cudaFuncSetAttribute(k_oz_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzSmem);
    if (e != cudaSuccess) return e;
    OzArgs p{};
    p.a = sa; p.b = sb; p.ea = ea; p.eb = eb;
    p.m = m; p.n = n; p.nkb = nkb; p.nrb_a = nrb_a; p.nrb_b = nrb_b;
    p.alpha = alpha; p.beta = beta; p.c = C; p.ldc = ldc; p.err = err;
    if (nrb_a > 65535) return cudaErrorInvalidValue;
    k_oz_gemm<<<dim3((unsigned)nrb_b, (unsigned)nrb_a), 128, kOzSmem, st>>>(p);
    count_launch();
    return cudaGetLastError();
}

} // namespace gci
