// chol_kernels.cu -- device kernels of the two-step Cholesky driver:
// candidate compression, the batch pivot search, the downdate of the
// diagonal and the reshaping kernels of the AO->MO transformation.
#include "gci_common.h"
#include "gci_runtime.h"
#include <cfloat>

namespace gci {

// Max of D over each shell pair's orbital-pair segment (DefineCandidates /
// DefineBatch, TwoStepCholesky_Step1.f90:547-552,600-605).
__global__ void k_segmax(const double* __restrict__ D, const int64_t* __restrict__ loc,
                         const int* __restrict__ dim, int64_t n, double* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double* d = D + loc[i];
        double m = -DBL_MAX;
        for (int k = 0; k < dim[i]; ++k) m = fmax(m, d[k]);
        out[i] = m;
    }
}

// new[i + ldn*j] = old[src[i] + ldo*j], i < nrows, j < ncols (chol2_Compress).
__global__ void k_gather_rows(const double* __restrict__ src_mat, int64_t ld_src, const int64_t* __restrict__ src,
                              int64_t nrows, int64_t ncols, double* __restrict__ dst, int64_t ld_dst)
{
    const int64_t total = nrows * ncols;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / nrows, i = t - j * nrows;
        dst[i + ld_dst * j] = src_mat[src[i] + ld_src * j];
    }
}

// dst[r + ld_dst*j] = src[r + ld_src*cols[j]] (pivot columns of M)
__global__ void k_gather_cols(const double* __restrict__ src, int64_t ld_src, const int* __restrict__ cols,
                              int64_t nrows, int64_t ncols, double* __restrict__ dst, int64_t ld_dst)
{
    const int64_t total = nrows * ncols;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / nrows, r = t - j * nrows;
        dst[r + ld_dst * j] = src[r + ld_src * cols[j]];
    }
}

__device__ __forceinline__ bool better(double v, int i, double bv, int bi)
{
    return v > bv || (v == bv && i < bi);
}

// Block-wide argmax with the reference's tie rule: strict '>' scanning in
// increasing index order, i.e. the largest value at the smallest index
// (chol2_BatchMax, TwoStepCholesky_Step1.f90:720-727).
__device__ void block_argmax(const double* __restrict__ v, int n, double& bestv, int& besti,
                             double* s_v, int* s_i)
{
    double bv = -DBL_MAX;
    int bi = 0x7fffffff;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (better(v[i], i, bv, bi)) { bv = v[i]; bi = i; }
    for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, bv, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { s_v[warp] = bv; s_i[warp] = bi; }
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        bv = lane < nw ? s_v[lane] : -DBL_MAX;
        bi = lane < nw ? s_i[lane] : 0x7fffffff;
        for (int off = 16; off > 0; off >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, off);
            const int oi = __shfl_down_sync(0xffffffffu, bi, off);
            if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
        }
        if (lane == 0) { s_v[0] = bv; s_i[0] = bi; }
    }
    __syncthreads();
    bestv = s_v[0];
    besti = s_i[0];
    __syncthreads();
}

// Micro-iterations of one macro iteration (chol2_Pivots, Step1.f90:1025-1064)
// restricted to the batch: the pivot choice depends only on the batch rows
// of M and of the new vectors, so the sequential part runs in one CTA on the
// nb x nb block Mbb; the vectors over all candidates follow afterwards as one
// triangular solve.  Lb(:, j) = (Mbb(:, piv_j) - Lb Lb(piv_j, :)^T) / sqrt(Dmax_j).
__global__ void __launch_bounds__(1024) k_pivot_batch(const double* __restrict__ Mbb, int nb, double* __restrict__ Db,
                                                      double* __restrict__ Lb, int* __restrict__ piv,
                                                      double* __restrict__ pdmax, int* __restrict__ npiv_out,
                                                      int64_t nchol0, int64_t maxnchol, double dmin)
{
    extern __shared__ double sh[];
    double* prow = sh;                                   // nb
    double* s_v = sh + nb;                               // 32
    int* s_i = reinterpret_cast<int*>(s_v + 32);         // 32
    double maxv; int maxi;
    block_argmax(Db, nb, maxv, maxi, s_v, s_i);
    int j = 0;
    bool go = (nchol0 < maxnchol) && nb > 0;
    while (go) {
        if (threadIdx.x == 0) { piv[j] = maxi; pdmax[j] = maxv; }
        for (int i = threadIdx.x; i < j; i += blockDim.x) prow[i] = Lb[maxi + (int64_t)nb * i];
        __syncthreads();
        const double sq = sqrt(maxv);
        for (int r = threadIdx.x; r < nb; r += blockDim.x) {
            double s = Mbb[r + (int64_t)nb * maxi];
            for (int i = 0; i < j; ++i) s -= Lb[r + (int64_t)nb * i] * prow[i];
            const double l = s / sq;
            Lb[r + (int64_t)nb * j] = l;
            Db[r] -= l * l;
        }
        __syncthreads();
        ++j;
        block_argmax(Db, nb, maxv, maxi, s_v, s_i);
        if (maxv <= dmin) go = false;
        if (j == nb || nchol0 + j == maxnchol) go = false;
    }
    if (threadIdx.x == 0) *npiv_out = j;
}

// Lp(j, i) = Lb(piv[j], i): the pivot rows of the new vectors (lower triangular)
__global__ void k_gather_pivrows(const double* __restrict__ Lb, int nb, const int* __restrict__ piv, int npiv,
                                 double* __restrict__ Lp)
{
    const int64_t total = (int64_t)npiv * npiv;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / npiv), jr = (int)(t - (int64_t)i * npiv);
        Lp[jr + (int64_t)npiv * i] = (i <= jr) ? Lb[piv[jr] + (int64_t)nb * i] : 0.0;
    }
}

// Inverse of a lower-triangular n x n matrix, one block per column
// (forward substitution with a block reduction per row).
__global__ void k_tri_inv_lower(const double* __restrict__ L, int n, double* __restrict__ X)
{
    __shared__ double red[32];
    __shared__ double xcol_s;
    for (int c = blockIdx.x; c < n; c += gridDim.x) {
        double* xc = X + (int64_t)n * c;
        for (int i = threadIdx.x; i < c; i += blockDim.x) xc[i] = 0.0;
        if (threadIdx.x == 0) xc[c] = 1.0 / L[c + (int64_t)n * c];
        __syncthreads();
        for (int i = c + 1; i < n; ++i) {
            double s = 0.0;
            for (int k = c + threadIdx.x; k < i; k += blockDim.x) s += L[i + (int64_t)n * k] * xc[k];
            for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0.0;
                for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) t += red[w];
                xcol_s = -t / L[i + (int64_t)n * i];
                xc[i] = xcol_s;
            }
            __syncthreads();
        }
    }
}

// D[r] -= sum_j L[r + ld*j]^2  (D(:) = D(:) - Lpqj(:,j)**2, Step1.f90:1046)
__global__ void k_downdate(double* __restrict__ D, const double* __restrict__ L, int64_t ld, int64_t n, int ncols)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double d = D[r];
        for (int j = 0; j < ncols; ++j) {
            const double l = L[r + ld * j];
            d -= l * l;
        }
        D[r] = d;
    }
}

__global__ void k_max(const double* __restrict__ v, int64_t n, double* __restrict__ out)
{
    __shared__ double red[32];
    double m = -DBL_MAX;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, v[i]);
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = -DBL_MAX;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) t = fmax(t, red[w]);
        *out = t;
    }
}

__global__ void k_zero_upper(double* __restrict__ A, int64_t n)
{
    const int64_t total = n * n;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / n, i = t - j * n;
        if (i < j) A[t] = 0.0;
    }
}

// Unpack Rkpq(k, pq) (k in [k0, k0+kc)) into the dense symmetric AO-pair
// layout U[p][q][k - k0] (both triangles) for the AO->MO GEMMs.
// One entry per stored orbital pair: pq_ao[2*i] = p, pq_ao[2*i+1] = q, and
// pq_col[i] = column of the pair in the (NVecs x MaxSubsetDim x NSubsets) array.
__global__ void k_unpack_rkpq(const double* __restrict__ R, int64_t nvecs, const int64_t* __restrict__ pq_col,
                              const int* __restrict__ pq_ao, int64_t npq, int64_t k0, int64_t kc, int64_t nao,
                              double* __restrict__ U)
{
    const int64_t total = npq * kc;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / kc, k = t - i * kc;
        const double v = R[(k0 + k) + nvecs * pq_col[i]];
        const int64_t p = pq_ao[2 * i], q = pq_ao[2 * i + 1];
        U[(p * nao + q) * kc + k] = v;
        if (p != q) U[(q * nao + p) * kc + k] = v;
    }
}

static inline unsigned grid_for(int64_t n, int threads, int64_t cap = 148LL * 32)
{
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

cudaError_t launch_segmax(const double* D, const int64_t* loc, const int* dim, int64_t n, double* out, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_segmax<<<grid_for(n, 256), 256, 0, s>>>(D, loc, dim, n, out);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_gather_rows(const double* src, int64_t lds, const int64_t* idx, int64_t nrows, int64_t ncols,
                               double* dst, int64_t ldd, cudaStream_t s)
{
    if (nrows <= 0 || ncols <= 0) return cudaSuccess;
    k_gather_rows<<<grid_for(nrows * ncols, 256), 256, 0, s>>>(src, lds, idx, nrows, ncols, dst, ldd);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_gather_cols(const double* src, int64_t lds, const int* cols, int64_t nrows, int64_t ncols,
                               double* dst, int64_t ldd, cudaStream_t s)
{
    if (nrows <= 0 || ncols <= 0) return cudaSuccess;
    k_gather_cols<<<grid_for(nrows * ncols, 256), 256, 0, s>>>(src, lds, cols, nrows, ncols, dst, ldd);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_pivot_batch(const double* Mbb, int nb, double* Db, double* Lb, int* piv, double* pdmax,
                               int* npiv, int64_t nchol0, int64_t maxnchol, double dmin, cudaStream_t s)
{
    const size_t smem = sizeof(double) * (size_t)(nb + 32) + sizeof(int) * 32;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_pivot_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_pivot_batch<<<1, 1024, smem, s>>>(Mbb, nb, Db, Lb, piv, pdmax, npiv, nchol0, maxnchol, dmin);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_gather_pivrows(const double* Lb, int nb, const int* piv, int npiv, double* Lp, cudaStream_t s)
{
    if (npiv <= 0) return cudaSuccess;
    k_gather_pivrows<<<grid_for((int64_t)npiv * npiv, 256), 256, 0, s>>>(Lb, nb, piv, npiv, Lp);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_tri_inv_lower(const double* L, int n, double* X, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_tri_inv_lower<<<n < 148 * 8 ? n : 148 * 8, 128, 0, s>>>(L, n, X);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_downdate(double* D, const double* L, int64_t ld, int64_t n, int ncols, cudaStream_t s)
{
    if (n <= 0 || ncols <= 0) return cudaSuccess;
    k_downdate<<<grid_for(n, 256), 256, 0, s>>>(D, L, ld, n, ncols);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_max(const double* v, int64_t n, double* out, cudaStream_t s)
{
    k_max<<<1, 1024, 0, s>>>(v, n, out);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_zero_upper(double* A, int64_t n, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_zero_upper<<<grid_for(n * n, 256), 256, 0, s>>>(A, n);
    count_launch();
    return cudaGetLastError();
}
cudaError_t launch_unpack_rkpq(const double* R, int64_t nvecs, const int64_t* pq_col, const int* pq_ao, int64_t npq,
                               int64_t k0, int64_t kc, int64_t nao, double* U, cudaStream_t s)
{
    if (npq <= 0 || kc <= 0) return cudaSuccess;
    k_unpack_rkpq<<<grid_for(npq * kc, 256), 256, 0, s>>>(R, nvecs, pq_col, pq_ao, npq, k0, kc, nao, U);
    count_launch();
    return cudaGetLastError();
}

} // namespace gci
