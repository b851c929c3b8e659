// gci_runtime.h -- host-side declarations of the kernel launchers.
#pragma once
#include "gci_common.h"

namespace gci {

// Number of kernels this library has launched (all launchers count themselves).
void count_launch(int64_t n = 1);
int64_t launches();

cudaError_t eri_module_init();
cudaError_t eri_launch(int tb, int tk, const EriArgs& args, cudaStream_t st);
// Kernel variant of the canonical class (tb, tk): 0 team kernel, 1..3
// ket-first kernel with 32, 64 or 128 lanes per quartet (only where built);
// eri_set_variant returns -1 when unavailable.
int eri_num_variants();
int eri_variant(int tb, int tk);
int eri_set_variant(int tb, int tk, int variant);
cudaError_t pair_records_launch(const ShellPairDev* pairs, int npairs, const double* xyz, const int* poff,
                                const double* exps, const double* coefs, const int* plist, double* pp,
                                cudaStream_t st);
// Hermite-matrix ERI path (eri_hermite.cuh, eri_hm_vectors.cu): row vectors of
// the listed pairs at offsets off[id], column vectors of the chunks, and the
// product kernel of row level L1, column level L2 and nt column tiles.
cudaError_t hm_rowvec_launch(const int* ids, int nids, const ShellPairDev* pairs, const double* pp,
                             const int64_t* off, const double* tmat, const int* toff, const int* nfunc, double* vec,
                             cudaStream_t st);
cudaError_t hm_colvec_launch(const HmChunk* chunks, int nchunks, const ShellPairDev* pairs, const double* pp,
                             const int* colfun, const double* tmat, const int* toff, const int* nfunc, double* vec,
                             cudaStream_t st);
cudaError_t hm_launch(int L1, int L2, int nt, const HmArgs& a, cudaStream_t st);
// Split-precision FP64 GEMM on the int8 tensor cores (ozaki_gemm.cu):
// C = alpha A B^T + beta C with A(i, l) = A[i ars + l als], B(j, l) = B[j brs + l bls],
// k <= ozaki_max_k(); `work` holds ozaki_workspace_bytes(m, n, k); `err` is set to 1
// when a bounded wait of the GEMM kernel expires.
size_t ozaki_workspace_bytes(int64_t m, int64_t n, int64_t k);
int64_t ozaki_max_k();
cudaError_t ozaki_dgemm_nt(int64_t m, int64_t n, int64_t k, double alpha, const double* A, int64_t ars, int64_t als,
                           const double* B, int64_t brs, int64_t bls, double beta, double* C, int64_t ldc,
                           void* work, int* err, cudaStream_t st);
// FP64 dense kernels on the DMMA tensor path (dense_fp64.cu).
// dgemm: C(i, j) = alpha sum_l A(i, l) B(l, j) + beta C(i, j) with A(i, l) = a[i sai + l sal],
// B(l, j) = b[l sbl + j sbj], C(i, j) = c[i sci + j scj] (+ batch strides sab, sbb, scb per
// batch index).  The flags declare structure whose zero part is skipped: kDgALower
// (A(i, l) = 0 for l > i), kDgBLower (B(l, j) = 0 for l < j), kDgBUpper (B(l, j) = 0 for
// l > j), kDgCLower (only C(i, j) with j <= i is written).  C must not overlap A or B.
constexpr int kDgALower = 1, kDgBLower = 2, kDgBUpper = 4, kDgCLower = 8;
struct DgemmArgs {
    int64_t m, n, k;
    double alpha, beta;
    const double* a;
    int64_t sai, sal, sab;
    const double* b;
    int64_t sbl, sbj, sbb;
    double* c;
    int64_t sci, scj, scb;
    int flags;
};
cudaError_t dgemm(const DgemmArgs& p, int64_t batch, cudaStream_t st);
// L (lower part of a, in place) and x = L^-1 (n x n, zeros above the diagonal) of the SPD
// matrix a (lower part read), both column-major with leading dimension ld; *info = j + 1 for
// the first non-positive pivot j found, else 0 (read it after the stream completes).  The
// upper triangle of a is used as scratch.
cudaError_t potrf_inverse(int64_t n, double* a, double* x, int64_t ld, int* info, cudaStream_t st);
// b (rows x w, leading dimension ldb) <- b l^-T for the w x w lower-triangular l (ldl).
cudaError_t trsm_rlt(int64_t rows, int64_t w, double* b, int64_t ldb, const double* l, int64_t ldl, cudaStream_t st);
cudaError_t boys_eval_launch(int m, int64_t n, const double* x, const double* table, double* out, cudaStream_t st);

cudaError_t launch_segmax(const double* D, const int64_t* loc, const int* dim, int64_t n, double* out, cudaStream_t s);
cudaError_t launch_gather_rows(const double* src, int64_t lds, const int64_t* idx, int64_t nrows, int64_t ncols,
                               double* dst, int64_t ldd, cudaStream_t s);
cudaError_t launch_gather_cols(const double* src, int64_t lds, const int* cols, int64_t nrows, int64_t ncols,
                               double* dst, int64_t ldd, cudaStream_t s);
cudaError_t launch_pivot_batch(const double* Mbb, int nb, double* Db, double* Lb, int* piv, double* pdmax,
                               int* npiv, int64_t nchol0, int64_t maxnchol, double dmin, cudaStream_t s);
cudaError_t launch_gather_pivrows(const double* Lb, int nb, const int* piv, int npiv, double* Lp, cudaStream_t s);
cudaError_t launch_tri_inv_lower(const double* L, int n, double* X, cudaStream_t s);
cudaError_t launch_downdate(double* D, const double* L, int64_t ld, int64_t n, int ncols, cudaStream_t s);
cudaError_t launch_max(const double* v, int64_t n, double* out, cudaStream_t s);
cudaError_t launch_zero_upper(double* A, int64_t n, cudaStream_t s);
cudaError_t launch_unpack_rkpq(const double* R, int64_t nvecs, const int64_t* pq_col, const int* pq_ao, int64_t npq,
                               int64_t k0, int64_t kc, int64_t nao, double* U, cudaStream_t s);

// adjoint path (grad_kernels.cu)
cudaError_t grad_module_init();
cudaError_t grad_pair_vectors_launch(const ShellPairDev* pairs, int npairs, const int64_t* gbase,
                                     const int* level_beg, const int* level_n, const int64_t* vec_off,
                                     const int64_t* hk_off, const double* xyz, const int* poff, const double* exps,
                                     const double* coefs, const int* plist, const double* tmat, const int* toff,
                                     const int* nfunc, const int* loc, const double* D, int64_t ldd, double* mP,
                                     double* mX, double* mY, double* mZ, double* vecs, double* hk, int* ppair,
                                     cudaStream_t st);
cudaError_t grad_potential_launch(int L1, int L2, const GradPotArgs& a, cudaStream_t st);
cudaError_t grad_dots_launch(int64_t beg, int64_t n, int HB, const double* vecs, const double* V, double* out,
                             cudaStream_t st);
cudaError_t grad_coulomb_matrix_launch(const ShellPairDev* pairs, int npairs, const int64_t* gbase,
                                       const int* level_beg, const int64_t* pot_off, const double* V, const double* pp,
                                       const double* tmat, const int* toff, const int* nfunc, const int* loc,
                                       double* J, int64_t ldj, cudaStream_t st);

} // namespace gci
