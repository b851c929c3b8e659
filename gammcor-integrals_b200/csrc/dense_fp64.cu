// dense_fp64.cu -- the FP64 dense linear algebra of the decomposition on the
// FP64 tensor cores (mma.sync m8n8k4 f64, the DMMA instruction of sm_100a):
//
//  * k_dgemm: C = alpha A B + beta C with element strides for every operand
//    (A(i, l) = a[i sai + l sal], B(l, j) = b[l sbl + j sbj], C(i, j) =
//    c[i sci + j scj]), an optional batch index, and structure flags that skip
//    the zero half of a triangular operand (the K range of a tile shrinks) or
//    the strictly upper tiles of a symmetric update.  128 x 128 tiles, 8 warps
//    of 64 x 32, K in blocks of 16 through a three-stage ring of shared
//    buffers filled by cp.async (two blocks in flight during the products).
//  * k_potrf_leaf: Cholesky factor and inverse of one diagonal block of at
//    most 64 rows in shared memory.
//  * k_trsm_leaf: X = B L^-T for a block of at most 32 columns, one row of B
//    per thread, by forward substitution.
//
// Host drivers (recursive, GEMM-dominated):
//  * potrf_inverse: L and L^-1 of an SPD matrix (real_Cholesky +
//    real_LowerTriangularInverse, real_linalg.f90:39-72, i.e. dpotrf + dtrtri):
//    A = [A11 .; A21 A22] -> (L11, X11) recursively; L21 = A21 X11^T;
//    A22 -= L21 L21^T; (L22, X22) recursively; X21 = -X22 L21 X11.
//  * trsm_rlt: B <- B L^-T (the vectors of a pivot batch, chol2_Lj,
//    TwoStepCholesky_Step1.f90:859-881): B1 <- B1 L11^-T; B2 -= B1 L21^T;
//    B2 <- B2 L22^-T, substitution at the leaves (backward stable, no explicit
//    inverse of the pivot block).
#include "gci_runtime.h"

namespace gci {

constexpr int kDgBM = 128, kDgBN = 128, kDgBK = 16, kDgThreads = 256, kDgStages = 3;
// Shared K slice of one operand: [kDgBK][kDgLdR] when its contiguous global index is the row
// index (i or j), [128][kDgLdK] when it is l.  Both paddings make the fragment loads of a
// half-warp conflict-free.
constexpr int kDgLdR = kDgBM + 4, kDgLdK = kDgBK + 4;
constexpr int kDgTile = kDgBM * kDgLdK > kDgBK * kDgLdR ? kDgBM * kDgLdK : kDgBK * kDgLdR;   // doubles
constexpr int kDgSmem = kDgStages * 2 * kDgTile * (int)sizeof(double);
constexpr int kLeafN = 64, kLeafLd = kLeafN + 1;
constexpr int kTrsmW = 32;

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

// 8-byte asynchronous copy global -> shared; src_bytes = 0 writes zero (src is not read)
__device__ __forceinline__ void cp_async8(double* dst, const double* src, int src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}

// AK: A's contiguous global index is l (sal == 1), else i; BK: B's is l (sbl == 1), else j.
// Each operand is copied along its contiguous index into the matching shared layout.
template <bool AK, bool BK>
__global__ void __launch_bounds__(kDgThreads, 1) k_dgemm(const DgemmArgs p)
{
    extern __shared__ __align__(16) double dg_smem[];
    const int64_t m0 = (int64_t)blockIdx.x * kDgBM, n0 = (int64_t)blockIdx.y * kDgBN;
    if ((p.flags & kDgCLower) && n0 >= m0 + kDgBM) return;   // tile strictly above the diagonal
    const double* A = p.a + (int64_t)blockIdx.z * p.sab;
    const double* B = p.b + (int64_t)blockIdx.z * p.sbb;
    double* Cm = p.c + (int64_t)blockIdx.z * p.scb;
    int64_t klo = 0, khi = p.k;
    if (p.flags & kDgALower) khi = min(khi, m0 + kDgBM);   // A(i, l) = 0 for l > i
    if (p.flags & kDgBUpper) khi = min(khi, n0 + kDgBN);   // B(l, j) = 0 for l > j
    if (p.flags & kDgBLower) klo = max(klo, n0);           // B(l, j) = 0 for l < j
    const int64_t nkt = khi > klo ? (khi - klo + kDgBK - 1) / kDgBK : 0;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    // copy s of this thread: tile row r + s dr, tile k kq + s dk
    const int a_r = AK ? tid >> 4 : tid & 127, a_k = AK ? tid & 15 : tid >> 7;
    const int b_r = BK ? tid >> 4 : tid & 127, b_k = BK ? tid & 15 : tid >> 7;
    constexpr int a_dr = AK ? 16 : 0, a_dk = AK ? 0 : 2;
    constexpr int b_dr = BK ? 16 : 0, b_dk = BK ? 0 : 2;
    auto a_off = [](int r, int k) { return AK ? r * kDgLdK + k : k * kDgLdR + r; };
    auto b_off = [](int r, int k) { return BK ? r * kDgLdK + k : k * kDgLdR + r; };
    auto issue = [&](int64_t kt) {
        if (kt < nkt) {
            const int64_t k0 = klo + kt * kDgBK;
            double* as = dg_smem + (kt % kDgStages) * 2 * kDgTile;
            double* bs = as + kDgTile;
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                const int ra = a_r + s * a_dr, ka = a_k + s * a_dk;
                const int64_t i = m0 + ra, l = k0 + ka;
                const bool va = i < p.m && l < khi;
                cp_async8(as + a_off(ra, ka), va ? A + i * p.sai + l * p.sal : A, va ? 8 : 0);
                const int rb = b_r + s * b_dr, kb = b_k + s * b_dk;
                const int64_t j = n0 + rb, lb = k0 + kb;
                const bool vb = j < p.n && lb < khi;
                cp_async8(bs + b_off(rb, kb), vb ? B + lb * p.sbl + j * p.sbj : B, vb ? 8 : 0);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");   // one group per tile, empty past the end
    };

    double acc[8][4][2];
#pragma unroll
    for (int mt = 0; mt < 8; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;

#pragma unroll
    for (int s = 0; s < kDgStages - 1; ++s) issue(s);
#pragma unroll 1
    for (int64_t kt = 0; kt < nkt; ++kt) {
        asm volatile("cp.async.wait_group %0;" ::"n"(kDgStages - 2) : "memory");   // tile kt has landed
        __syncthreads();   // every thread's copies of tile kt; every warp done with tile kt - 1
        issue(kt + kDgStages - 1);
        const double* as = dg_smem + (kt % kDgStages) * 2 * kDgTile;
        const double* bs = as + kDgTile;
#pragma unroll
        for (int kk = 0; kk < kDgBK / 4; ++kk) {
            const int kq = kk * 4 + (lane & 3);
            double af[8], bf[4];
#pragma unroll
            for (int mt = 0; mt < 8; ++mt) af[mt] = as[a_off(wm * 64 + mt * 8 + (lane >> 2), kq)];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) bf[nt] = bs[b_off(wn * 32 + nt * 8 + (lane >> 2), kq)];
#pragma unroll
            for (int mt = 0; mt < 8; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt], af[mt], bf[nt]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");

    // D fragment: lane l holds D(l / 4, 2 (l % 4) + e)
#pragma unroll
    for (int mt = 0; mt < 8; ++mt) {
        const int64_t i = m0 + wm * 64 + mt * 8 + (lane >> 2);
        if (i >= p.m) continue;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int64_t j = n0 + wn * 32 + nt * 8 + 2 * (lane & 3) + e;
                if (j >= p.n || ((p.flags & kDgCLower) && j > i)) continue;
                double* cp = Cm + i * p.sci + j * p.scj;
                const double v = p.alpha * acc[mt][nt][e];
                *cp = p.beta == 0.0 ? v : fma(p.beta, *cp, v);
            }
    }
}

cudaError_t dgemm(const DgemmArgs& p, int64_t batch, cudaStream_t st)
{
    if (p.m <= 0 || p.n <= 0 || batch <= 0) return cudaSuccess;
    const int64_t gm = (p.m + kDgBM - 1) / kDgBM, gn = (p.n + kDgBN - 1) / kDgBN;
    if (gm > 0x7fffffffLL || gn > 65535 || batch > 65535) return cudaErrorInvalidValue;
    const bool ak = p.sal == 1 && p.sai != 1, bk = p.sbl == 1 && p.sbj != 1;
    auto fn = ak ? (bk ? k_dgemm<true, true> : k_dgemm<true, false>) : (bk ? k_dgemm<false, true> : k_dgemm<false, false>);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kDgSmem);
    if (e != cudaSuccess) return e;
    fn<<<dim3((unsigned)gm, (unsigned)gn, (unsigned)batch), kDgThreads, kDgSmem, st>>>(p);
    count_launch();
    return cudaGetLastError();
}

// ------------------------------------------------------------------ leaves
// Diagonal block [off, off + n) of a (n <= 64): L (lower part of a) and X = L^-1 (x, zeros
// above the diagonal).  A non-positive pivot j sets *info = off + j + 1 (first failure kept).
__global__ void __launch_bounds__(128) k_potrf_leaf(double* a, double* x, int64_t ld, int64_t off, int n, int* info)
{
    extern __shared__ double lf_smem[];
    double* S = lf_smem;                       // [kLeafN][kLeafLd]
    double* X = lf_smem + kLeafN * kLeafLd;    // [kLeafN][kLeafLd]
    const int tid = threadIdx.x;
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, j = idx / n;
        S[i * kLeafLd + j] = i >= j ? a[(off + i) + (off + j) * ld] : 0.0;
    }
    __syncthreads();
    for (int j = 0; j < n; ++j) {
        const double d = S[j * kLeafLd + j];   // the same value in every thread: a uniform branch
        if (!(d > 0.0)) {
            if (tid == 0) atomicCAS(info, 0, (int)(off + j + 1));
            return;
        }
        const double r = sqrt(d);
        __syncthreads();
        for (int i = j + tid; i < n; i += blockDim.x) S[i * kLeafLd + j] = i == j ? r : S[i * kLeafLd + j] / r;
        __syncthreads();
        const int t = n - j - 1;
        for (int idx = tid; idx < t * t; idx += blockDim.x) {
            const int i = j + 1 + idx % t, k = j + 1 + idx / t;
            if (k <= i) S[i * kLeafLd + k] -= S[i * kLeafLd + j] * S[k * kLeafLd + j];
        }
        __syncthreads();
    }
    // X = L^-1 column by column: X(c, c) = 1 / L(c, c), X(i, c) = -sum_{c <= k < i} L(i, k) X(k, c) / L(i, i)
    if (tid < n) {
        const int c = tid;
        X[c * kLeafLd + c] = 1.0 / S[c * kLeafLd + c];
        for (int i = c + 1; i < n; ++i) {
            double s = 0.0;
            for (int k = c; k < i; ++k) s = fma(S[i * kLeafLd + k], X[k * kLeafLd + c], s);
            X[i * kLeafLd + c] = -s / S[i * kLeafLd + i];
        }
    }
    __syncthreads();
    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, j = idx / n;
        if (i >= j) a[(off + i) + (off + j) * ld] = S[i * kLeafLd + j];
        x[(off + i) + (off + j) * ld] = i >= j ? X[i * kLeafLd + j] : 0.0;
    }
}

// B(r, 0..w) <- B(r, 0..w) L^-T for the w x w lower-triangular block L (w <= 32): row r of
// the solution satisfies sum_{i <= j} X(r, i) L(j, i) = B(r, j).
__global__ void __launch_bounds__(128) k_trsm_leaf(double* b, int64_t ldb, int64_t rows, const double* l, int64_t ldl,
                                                   int w)
{
    __shared__ double Ls[kTrsmW][kTrsmW + 1];
    for (int idx = threadIdx.x; idx < kTrsmW * kTrsmW; idx += blockDim.x) {
        const int i = idx % kTrsmW, k = idx / kTrsmW;
        Ls[i][k] = (i < w && k <= i) ? l[i + k * ldl] : 0.0;
    }
    __syncthreads();
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    double xv[kTrsmW];
#pragma unroll
    for (int j = 0; j < kTrsmW; ++j) {
        xv[j] = 0.0;
        if (j < w) {
            double s = b[r + j * ldb];
#pragma unroll
            for (int i = 0; i < j; ++i) s = fma(-Ls[j][i], xv[i], s);
            xv[j] = s / Ls[j][j];
            b[r + j * ldb] = xv[j];
        }
    }
}

// ------------------------------------------------------------------ drivers
static DgemmArgs dg(int64_t m, int64_t n, int64_t k, double alpha, const double* a, int64_t sai, int64_t sal,
                    const double* b, int64_t sbl, int64_t sbj, double beta, double* c, int64_t sci, int64_t scj,
                    int flags)
{
    DgemmArgs p{};
    p.m = m; p.n = n; p.k = k; p.alpha = alpha; p.beta = beta;
    p.a = a; p.sai = sai; p.sal = sal;
    p.b = b; p.sbl = sbl; p.sbj = sbj;
    p.c = c; p.sci = sci; p.scj = scj;
    p.flags = flags;
    return p;
}

static cudaError_t potrf_rec(double* a, double* x, int64_t ld, int64_t off, int64_t n, int* info, cudaStream_t st)
{
    if (n <= kLeafN) {
        k_potrf_leaf<<<1, 128, 2 * kLeafN * kLeafLd * sizeof(double), st>>>(a, x, ld, off, (int)n, info);
        count_launch();
        return cudaGetLastError();
    }
    const int64_t n1 = (n / 2 + kLeafN - 1) / kLeafN * kLeafN, n2 = n - n1;
    const int64_t o2 = off + n1;
    cudaError_t e;
    if ((e = potrf_rec(a, x, ld, off, n1, info, st)) != cudaSuccess) return e;
    double* A21 = a + o2 + off * ld;
    double* X11 = x + off + off * ld;
    double* X21 = x + o2 + off * ld;
    double* A22 = a + o2 + o2 * ld;
    double* X22 = x + o2 + o2 * ld;
    double* A12 = a + off + o2 * ld;   // upper triangle of this block: T = L21 X11, stored transposed
    // L21 = A21 X11^T, held in X21 until L22 is done
    if ((e = dgemm(dg(n2, n1, n1, 1.0, A21, 1, ld, X11, ld, 1, 0.0, X21, 1, ld, kDgBUpper), 1, st)) != cudaSuccess)
        return e;
    // A22 -= L21 L21^T (lower tiles)
    if ((e = dgemm(dg(n2, n2, n1, -1.0, X21, 1, ld, X21, ld, 1, 1.0, A22, 1, ld, kDgCLower), 1, st)) != cudaSuccess)
        return e;
    if ((e = potrf_rec(a, x, ld, o2, n2, info, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpy2DAsync(A21, ld * sizeof(double), X21, ld * sizeof(double), n2 * sizeof(double), n1,
                               cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return e;
    // T = L21 X11 (X11 lower: B(l, j) = 0 for l < j), into A12 as T^T
    if ((e = dgemm(dg(n2, n1, n1, 1.0, A21, 1, ld, X11, 1, ld, 0.0, A12, ld, 1, kDgBLower), 1, st)) != cudaSuccess)
        return e;
    // X21 = -X22 T (X22 lower)
    return dgemm(dg(n2, n1, n2, -1.0, X22, 1, ld, A12, ld, 1, 0.0, X21, 1, ld, kDgALower), 1, st);
}

cudaError_t potrf_inverse(int64_t n, double* a, double* x, int64_t ld, int* info, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_potrf_leaf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         2 * kLeafN * kLeafLd * (int)sizeof(double));
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(info, 0, sizeof(int), st)) != cudaSuccess) return e;
    // the blocks above the diagonal of X are never written: they stay zero
    if ((e = cudaMemset2DAsync(x, ld * sizeof(double), 0, n * sizeof(double), n, st)) != cudaSuccess) return e;
    return potrf_rec(a, x, ld, 0, n, info, st);
}

static cudaError_t trsm_rec(int64_t rows, double* b, int64_t ldb, const double* l, int64_t ldl, int64_t c0, int64_t w,
                            cudaStream_t st)
{
    if (w <= kTrsmW) {
        const int64_t grid = (rows + 127) / 128;
        if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
        k_trsm_leaf<<<(unsigned)grid, 128, 0, st>>>(b + c0 * ldb, ldb, rows, l + c0 + c0 * ldl, ldl, (int)w);
        count_launch();
        return cudaGetLastError();
    }
    const int64_t w1 = (w / 2 + kTrsmW - 1) / kTrsmW * kTrsmW, w2 = w - w1;
    cudaError_t e;
    if ((e = trsm_rec(rows, b, ldb, l, ldl, c0, w1, st)) != cudaSuccess) return e;
    // B2 -= X1 L21^T: B'(q, j) = L(c0 + w1 + j, c0 + q)
    if ((e = dgemm(dg(rows, w2, w1, -1.0, b + c0 * ldb, 1, ldb, l + (c0 + w1) + c0 * ldl, ldl, 1, 1.0,
                      b + (c0 + w1) * ldb, 1, ldb, 0),
                   1, st)) != cudaSuccess)
        return e;
    return trsm_rec(rows, b, ldb, l, ldl, c0 + w1, w2, st);
}

cudaError_t trsm_rlt(int64_t rows, int64_t w, double* b, int64_t ldb, const double* l, int64_t ldl, cudaStream_t st)
{
    if (rows <= 0 || w <= 0) return cudaSuccess;
    return trsm_rec(rows, b, ldb, l, ldl, 0, w, st);
}

} // namespace gci
