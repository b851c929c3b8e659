/*
 * gci.h -- C ABI of the B200 integral-direct Cholesky ERI library
 * (libgci.so).  Plain pointers and sizes only; every call returns an int
 * status (0 = success, negative = error) and gci_last_error() gives the
 * message of the last failure on the calling thread.
 *
 * This is the drop-in boundary for the reference's Gammcor interface
 * (modrzejewski/gammcor-integrals, src/gammcor-interface/Cholesky_Gammcor.f90).
 * A Fortran ISO_C_BINDING shim keeping the module Cholesky_Gammcor and the
 * type TCholeskyVecsOTF binds these entry points
 * (gammcor-integrals_b200/fortran/cholesky_gammcor_gpu.f90).
 *
 * Conventions: arrays are column-major (Fortran order); indices passed in
 * arrays are 1-based exactly as in TAOBasis; integers are int64_t so that
 * both default-integer and -i8 builds of the caller can convert losslessly.
 */
#ifndef GCI_H
#define GCI_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define GCI_OK                 0
#define GCI_ERR_ARG           -1   /* invalid argument / dimension       */
#define GCI_ERR_CUDA          -2   /* CUDA runtime or kernel launch failure */
#define GCI_ERR_UNSUPPORTED   -3   /* angular momentum beyond the kernels, or a mode not built */
#define GCI_ERR_NOT_CONVERGED -4   /* MaxNCholesky reached unconverged    */
#define GCI_ERR_NOT_SPD       -5   /* pivot block V_JJ not positive definite */
#define GCI_ERR_BUFFER        -6   /* buffer too small                    */
#define GCI_ERR_NOMEM         -7   /* device allocation failed            */
#define GCI_ERR_STATE         -8   /* handle lacks the requested data     */

/* Accuracy levels: CHOL_ACCURACY_* of Cholesky_Gammcor.f90:14-17 */
#define GCI_ACCURACY_DEFAULT   1   /* tau = 1e-5  */
#define GCI_ACCURACY_TIGHT     2   /* tau = 1e-6  */
#define GCI_ACCURACY_LUDICROUS 3   /* tau = 1e-7  */
#define GCI_ACCURACY_DEBUG     4   /* tau = 1e-10 */

/* gci_rkpq flags */
#define GCI_FLAG_MATERIALIZE_RKPQ   1  /* store Rkpq on the device (otherwise Rkab is built from V(pq,J) directly) */
#define GCI_FLAG_PIVOT_DECODE_STORAGE 2 /* decode diagonal-shell-pair pivots in storage order (the reference decodes
                                          them with chol2_pq2p_ge_q, TwoStepCholesky_Step2.f90:422-466) */
#define GCI_FLAG_MIXED_STEP1        4  /* M - L L^T of the pivot search (chol2_SubtractR) as a split-precision
                                          GEMM on the int8 tensor cores (gci_dgemm_split) */

/* Precision of the AO->MO GEMMs: FP64 (DMMA tensor-core GEMM) or split precision on the int8
 * tensor cores (gci_dgemm_split) */
#define GCI_PREC_FP64   0
#define GCI_PREC_MIXED  1

/* Orbital orderings: ORBITAL_ORDERING_* of Auto2eInterface.f90:12-17 */
#define GCI_ORDERING_AUTO2E      0
#define GCI_ORDERING_MOLPRO      1
#define GCI_ORDERING_ORCA        2
#define GCI_ORDERING_DALTON      3
#define GCI_ORDERING_OPEN_MOLCAS 4
#define GCI_ORDERING_PYSCF       5

/* The arrays of TAOBasis (basis_definitions.f90:94-192) the path reads. */
typedef struct {
    int64_t natoms, nshells, nshellparams;
    int64_t ldprim;                  /* leading dim of cntr_coeffs/exponents (MaxNPrimitives) */
    int64_t ldnorm;                  /* leading dim of norm_factors */
    const double *atom_coords;       /* AtomCoords(3, NAtoms) */
    const int64_t *shell_centers;    /* ShellCenters(NShells), 1-based atom */
    const int64_t *shell_params_idx; /* ShellParamsIdx(NShells), 1-based */
    const int64_t *shell_momentum;   /* ShellMomentum(NShellParams) */
    const int64_t *nprimitives;      /* NPrimitives(NShellParams) */
    const double *cntr_coeffs;       /* CntrCoeffs(ldprim, NShellParams), primitive norms folded in */
    const double *exponents;         /* Exponents(ldprim, NShellParams) */
    const double *norm_factors;      /* NormFactorsSpher or NormFactorsCart(ldnorm, NShellParams) */
    int32_t spher_ao;                /* SpherAO */
} gci_basis;

typedef struct gci_handle gci_handle;

/* Library/device initialisation (auto2e_init + boys_init, Cholesky_Gammcor.f90:347-350).
 * Idempotent. */
int gci_init(void);

/* chol_gammcor_Rkpq (Cholesky_Gammcor.f90:335-377) + chol_gammcor_CoulombMatrix (:380-441):
 * two-step Cholesky (chol2_Algo_Koch_JCP2019, TwoStepCholesky.f90:45-71).  omega <= 0 means
 * the full-range Coulomb operator (Kappa = 0). */
int gci_rkpq(const gci_basis *basis, int accuracy, double omega, int flags, gci_handle **out);

/* gci_rkpq for many independent molecules at once (the reference decomposes one molecule per
 * chol_gammcor_Rkpq call, Cholesky_Gammcor.f90:335-377).  The molecules are taken largest
 * first from one queue by nstreams host workers (<= 0: 16; at most 64), each with its own
 * CUDA stream, so that the kernels of different molecules run
 * concurrently on the GPU.  out[i] receives the handle of bases[i] (same results as gci_rkpq
 * on that basis).  On an error no handle is returned (all out[i] = NULL) and
 * gci_last_error() names the lowest-index molecule that failed.  Batch calls from
 * different caller threads run one after another. */
int gci_rkpq_batch(int64_t nmol, const gci_basis *bases, int accuracy, double omega, int flags, int nstreams,
                   gci_handle **out);

/* Dimensions of TCholeskyVecsOTF / TChol2Vecs (TwoStepCholesky_definitions.f90:56-74). */
int gci_query(const gci_handle *h, int64_t *nvecs, int64_t *max_subset_dim, int64_t *nsubsets,
              int64_t *norbpairs, int64_t *nshellpairs, int64_t *npivshellpairs);

/* Rkpq(NVecs, MaxSubsetDim, NSubsets) -> host, column-major (TCholeskyVecsOTF%Rkpq). */
int gci_copy_rkpq(const gci_handle *h, double *dst);

/* Chol2Data arrays (TChol2Vecs), 1-based indices as the Fortran type holds them.
 * Any pointer may be NULL.  Sizes: shellpairs 2 x NShellPairs, shellpairloc 3 x NShellPairs,
 * shellpairdim NShellPairs, subsetdim/subsetbounds(2x) NSubsets, pivots NOrbPairs,
 * pivotshellpairs/loc/dim NPivotShellPairs, pivotorbpairs NVecs, inv_l NVecs x NVecs. */
int gci_copy_chol2data(const gci_handle *h, int64_t *shellpairs, int64_t *shellpairloc, int64_t *shellpairdim,
                       int64_t *subsetdim, int64_t *subsetbounds, int64_t *pivots, int64_t *pivotshellpairs,
                       int64_t *pivotshellpairloc, int64_t *pivotshellpairdim, int64_t *pivotorbpairs,
                       double *inv_l);

/* Columns R(:, pq) of the Cholesky vectors for n orbital pairs (FULL-storage indices,
 * 1-based, repeats allowed) without materialising Rkpq: the full-dimension integrals of
 * those pairs against the pivot columns (chol2_Vabrs, TwoStepCholesky_Step2.f90:242-419,
 * restricted to their shell pairs) times Inv_L (chol2_FullDimVectors_Batch,
 * TwoStepCholesky.f90:378-416).  out: NVecs x n, column-major, host memory. */
int gci_rkpq_columns(gci_handle *h, int64_t n, const int64_t *pq, double *out);

/* Pivot sequence of step 1 (FULL-storage orbital-pair indices, 1-based, selection order)
 * and the residual diagonal at each selection.  Either pointer may be NULL. */
int gci_pivot_order(const gci_handle *h, int64_t *order, double *dmax);

/* chol_gammcor_Rkab (Cholesky_Gammcor.f90:26-92) after the AO-order conversion done by
 * the caller (auto2e_interface_AngFuncTransf): CA(ldca, *), CB(ldcb, *) in Auto2e AO order,
 * columns a0..a1 and b0..b1 (1-based inclusive).  Rkab(NVecs, NA*NB), k fastest, then a,
 * then b.  max_buffer_mb bounds the AO->MO work buffers (MaxBufferDimMB). */
int gci_rkab(gci_handle *h, const double *CA, int64_t ldca, int64_t a0, int64_t a1,
             const double *CB, int64_t ldcb, int64_t b0, int64_t b1, int64_t max_buffer_mb,
             int precision, double *rkab);

/* gci_rkab with CA, CB and Rkab in device memory (no host copies); same layout. */
int gci_rkab_device(gci_handle *h, const double *CA, int64_t ldca, int64_t a0, int64_t a1,
                    const double *CB, int64_t ldcb, int64_t b0, int64_t b1, int64_t max_buffer_mb,
                    int precision, double *rkab);

/* Work done on this handle: [0..4] GEMM flops of M-LL^T, new vectors, potrf+trtri, Inv_L
 * products, AO->MO; [5] shell quartets, [6] primitive quartets, [7] integrals evaluated;
 * then per canonical class (bra type, ket type) of 10 x 10 pair types, 6 counters:
 * quartets, primitive quartets after the primitive-pair screen, integrals, primitive
 * quartets before that screen, bra primitive pairs x quartets, ket primitive pairs x
 * quartets.
 * Pair type of (l_hi, l_lo) = l_hi(l_hi+1)/2 + l_lo. */
int gci_stats(const gci_handle *h, double *out, int n);

/* Kernels of this library launched so far in the process. */
int gci_kernel_launches(int64_t *n);

/* The CUDA stream (cudaStream_t) every call of the library runs on. */
int gci_get_stream(void **stream);

/* Per-phase device times (seconds) of the last gci_rkpq/gci_rkab on this handle:
 * [0] Vdiag [1] step-1 ERI (time_2e) [2] M - L L^T (time_rTr) [3] pivots + vectors (time_rk)
 * [4] compress [5] V_JJ ERI [6] potrf+trtri [7] full-dim ERI [8] Inv_L GEMM [9] AO->MO GEMMs
 * [10] step-1 macro iterations (count) [11] total rkpq wall [12] total rkab wall. */
int gci_timings(const gci_handle *h, double *out, int n);

void gci_free(gci_handle *h);
const char *gci_last_error(void);

/* ---- kernel-level entry points (no reference counterpart beyond the cited routine) ---- */

/* Boys function on the device: out[i*(m+1)+k] = F_k(x[i]), k = 0..m (fm, boys.f90:224-281). */
int gci_boys(int m, int64_t n, const double *x, double *out);

/* Real-solid-harmonic coefficients, (2L+1) x ncart(L) row-major, m = -L..L
 * (AutoSpherTransf.py:147-160 as used by auto2e_SpherTransf.f90). Host only. */
int gci_spher_coeffs(int L, double *U);

/* basis_NormalizeCntrCoeffs (basis_sets.f90:894-945) in place + SpherGTO_NormFactors
 * (sphergto.f90:166-211).  Host only. */
int gci_normalize_basis(int64_t nparams, int64_t ldprim, const int64_t *L, const int64_t *nprim,
                        const double *exps, double *coefs, double *norm_cart, int64_t ldcart,
                        double *norm_spher, int64_t ldsph);

/* Every shell-pair x shell-pair ERI block (pq|rs) of a basis: out is NPQ x NPQ, column-major,
 * with orbital pairs in the chol2_Vdiag order (ShB outer, ShA >= ShB inner; a fastest, lower
 * triangle for ShA == ShB).  Small bases only (tests). */
int gci_eri_pairs(const gci_basis *basis, double omega, double *out, int64_t ld);

/* ---- ERI kernel selection (no counterpart in the reference) ---- */

/* Each ERI class (pair types tb >= tk, pair type = lhi*(lhi+1)/2 + llo of the
 * two shells' angular momenta) has a team kernel (variant 0: lanes over the
 * ket Hermite indices; bra types up to (d,d)) and, for bra types from (d,s) up,
 * ket-first kernels with 32, 64 or 128 lanes per quartet (variants 1, 2, 3,
 * where built).  gci_eri_variant(tb, tk, v): v >= 0 selects, v < 0 only
 * queries; returns the variant in use (>= 0) or GCI_ERR_ARG.  The choice is
 * process-wide. */
int gci_eri_variant(int tb, int tk, int variant);

/* Split-precision FP64 GEMM on the int8 tensor cores (no counterpart in the reference; the
 * split-precision form of its dgemm calls, real_linalg.f90:1331-1361): C = alpha A B^T + beta C
 * with A (m x k), B (n x k), C (m x n) column-major DEVICE pointers on the library's stream.
 * Each row of A and B is scaled by a power of two and cut into seven 8-bit slices (Ozaki
 * splitting); the 34 slice products with s + t <= 9 run as tcgen05 int8 MMAs with exact int32
 * accumulation and are recombined in FP64.  Error ~1e-12 of max|A_i| max|B_j| for k = 16k. */
int gci_dgemm_split(int64_t m, int64_t n, int64_t k, double alpha, const double *A, int64_t lda,
                    const double *B, int64_t ldb, double beta, double *C, int64_t ldc);

/* ---- FP64 dense kernels of the decomposition (DMMA tensor cores, mma.sync m8n8k4 f64) ----
 * Like gci_dgemm_split these run on the library's stream (gci_get_stream), which does not wait
 * for the caller's streams: the inputs must be complete before the call.  They return after
 * the results are complete. */

/* C = alpha A B^T + beta C in FP64, same argument convention as gci_dgemm_split (the
 * dgemm("N", "T", ...) calls of real_linalg.f90:1331-1361, e.g. chol2_SubtractR,
 * TwoStepCholesky_Step1.f90:628-691).  DEVICE pointers, library stream. */
int gci_dgemm(int64_t m, int64_t n, int64_t k, double alpha, const double *A, int64_t lda, const double *B,
              int64_t ldb, double beta, double *C, int64_t ldc);

/* real_Cholesky + real_LowerTriangularInverse (real_linalg.f90:39-72, dpotrf("L") then
 * dtrtri("L", "N")): A (n x n, lda, lower triangle read) is overwritten by L in its lower
 * triangle (its upper triangle is used as scratch); X (n x n, ldx = lda) receives L^-1 with
 * zeros above the diagonal.  DEVICE pointers.  GCI_ERR_NOT_SPD when a pivot is not
 * positive (the reference stops with "Cholesky factorization failed"). */
int gci_cholesky_inverse(int64_t n, double *A, int64_t lda, double *X);

/* B (rows x w, ldb) <- B L^-T for the w x w lower-triangular L (ldl): dtrsm("R", "L", "T",
 * "N") as used for the vectors of a pivot batch (chol2_Lj, TwoStepCholesky_Step1.f90:859-881).
 * DEVICE pointers. */
int gci_trsm_rlt(int64_t rows, int64_t w, double *B, int64_t ldb, const double *L, int64_t ldl);

/* Hermite-matrix ERI kernels (default on).  For spherical bases the
 * product-mode stages (step-1 pivot columns, the pivot block, the
 * full-dimension stage, gci_eri_pairs) contract each pair's primitive
 * Hermite coefficients with the normalised solid-harmonic transforms once,
 * and evaluate every primitive quartet as dense FP64 tensor-core products
 * (the columns a stage keeps times the Hankel matrix R(h + g)).  The class
 * kernels above remain for the diagonal stage and Cartesian bases.
 * enable: 1 on, 0 off, 2 on with per-class timing (the class launches then
 * run one after another, each timed with CUDA events), < 0 query only;
 * returns the previous setting.  Process-wide. */
int gci_eri_hm(int enable);

/* Work of the Hermite-matrix kernels of a decomposition (and its gci_rkab
 * calls): for every row level L1 (0..6), column level L2 (0..6) and column
 * tile count (1..7, at most 7 for L1 <= 3, 5 for L1 = 4, 4 for L1 = 5, 3 for L1 = 6), in that
 * order: launches, device seconds (measured only with gci_eri_hm(2)) and
 * tensor-core flops issued (padding included); 7 x 7 x 7 x 3 values. */
int gci_eri_hm_stats(const gci_handle *h, double *out, int n);

/* Autotuner: times every variant of every class that occurs in `basis` on a
 * product-mode sample of its shell pairs (up to max_pairs bra and max_pairs
 * ket pairs per class) with CUDA events and keeps the fastest.  If
 * `seconds` is not NULL it receives 10 x 10 x 4 launch times (tb, tk,
 * variant; 0 where not measured). */
int gci_autotune_eri(const gci_basis *basis, int max_pairs, double *seconds);

/* ---- adjoint: Coulomb energy and nuclear gradient (no counterpart in the reference) ---- */

/* J = 1/2 sum_{pq,rs} D_pq (pq|rs) D_rs of a density D(ldd, NAO) (column-major, AO order of
 * the basis; D is symmetrised) and its derivatives, from derivative integrals built by Hermite
 * index shifts of the reference's McMurchie-Davidson scheme (E coefficients
 * auto2e_Hermite.f90:10-423, R_tuv :425-11878, Boys boys.f90:224-281):
 *   energy  J (may be NULL)
 *   grad    dJ/dAtomCoords, 3 x NAtoms column-major (may be NULL)
 *   jmat    Coulomb matrix J_pq = sum_rs (pq|rs) D_rs = dJ/dD_pq, ldj x NAO (may be NULL).
 * omega <= 0: full-range Coulomb operator. */
int gci_coulomb_grad(const gci_basis *basis, double omega, const double *D, int64_t ldd, double *energy,
                     double *grad, double *jmat, int64_t ldj);

/* gci_coulomb_grad with D and jmat in device memory (energy and grad stay host pointers). */
int gci_coulomb_grad_device(const gci_basis *basis, double omega, const double *D_dev, int64_t ldd,
                            double *energy, double *grad, double *jmat_dev, int64_t ldj);

/* Primitive quartets evaluated by the last gci_coulomb_grad* call, per (bra level, ket level)
 * of shell-pair Hermite levels lA+lB: out[L1 * 7 + L2], up to n entries (49). */
int gci_coulomb_grad_work(double *out, int n);

/* ---- allocation-free entry point (no counterpart in the reference) ---- */

/* Size of the fixed device scratch behind gci_eri_pairs_noalloc: a file-scope
 * __device__ array that every GPU on which libgci.so's code is loaded holds
 * until the process exits. */
#define GCI_NOALLOC_SCRATCH_BYTES ((int64_t)16 << 20)

/* The same NPQ x NPQ ERI matrix as gci_eri_pairs, for callers that cannot
 * allocate device memory: host codes whose device memory is owned by another
 * allocator (a caching pool that has reserved the card, e.g. a framework's or a
 * Fortran host program's), and code paths that must not call cudaMalloc or
 * cudaFree because those calls synchronise the whole device.  This call makes
 * no cudaMalloc or cudaFree call and uses no allocating library routine; its
 * working data (Boys table, basis, shell-pair tables, primitive-pair records,
 * index maps) lives in the fixed scratch of GCI_NOALLOC_SCRATCH_BYTES.
 *
 *   out_dev  DEVICE pointer to ld x NPQ doubles (column-major), on the current
 *            device; every element of the NPQ columns is written (rows past NPQ
 *            are set to zero), orbital pairs in the gci_eri_pairs order.
 *   stream   cudaStream_t to work on (NULL: the legacy default stream).  The
 *            call returns after the stream has finished the work.
 *
 * A basis whose tables need more than GCI_NOALLOC_SCRATCH_BYTES is rejected
 * with GCI_ERR_BUFFER before any device work (use gci_eri_pairs for it).
 * The first call on a device looks up the scratch's device address on that
 * device (once per device, with it current); make that first call before any
 * stream capture.  All calls share the one scratch array, which keeps the last
 * call's contents: calls that overlap on the GPU (other threads, other streams
 * of the same device) race on it and must be serialised by the caller. */
int gci_eri_pairs_noalloc(const gci_basis *basis, double omega, double *out_dev, int64_t ld, void *stream);

#ifdef __cplusplus
}
#endif
#endif
