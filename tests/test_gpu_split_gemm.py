"""GPU tests of the split-precision path: gci_dgemm_split (int8 tensor-core
Ozaki splitting, tcgen05) against FP64 products, and the decomposition and
AO->MO transform with the split-precision GEMMs (GCI_FLAG_MIXED_STEP1,
GCI_PREC_MIXED) against the FP64 path and the oracle.

Tolerance of the GEMM: the splitting keeps ~49 bits of every row relative to
the row's largest element and drops slice products below 2^-63, so
|C - C_fp64| <= 1e-13 k max|A_i| max|B_j| (written per element below)."""
import ctypes as C

import numpy as np
import pytest

from gammcor_integrals_b200 import _capi, molecules
from gammcor_integrals_b200 import cholesky_gammcor as cg
from helpers import both
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _split_gemm(lib, A, B, Cm, alpha, beta):
    """A (m x k), B (n x k), C (m x n) as column-major torch tensors given by their
    transposes At (k x m), Bt (k x n), Ct (n x m)."""
    import torch
    k, m = A.shape
    n = B.shape[1]
    torch.cuda.synchronize()
    _capi.check(lib.gci_dgemm_split(m, n, k, alpha, C.c_void_p(A.data_ptr()), m, C.c_void_p(B.data_ptr()), n,
                                    beta, C.c_void_p(Cm.data_ptr()), m))
    torch.cuda.synchronize()


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (128, 64, 128), (300, 70, 1000), (1000, 129, 5000),
                                   (2000, 200, 17000)])
def test_split_gemm_matches_fp64(gpu_lib, m, n, k):
    import torch
    g = torch.Generator(device="cuda").manual_seed(m + 7 * n + 13 * k)
    At = torch.randn(k, m, dtype=torch.float64, device="cuda", generator=g)
    Bt = torch.randn(k, n, dtype=torch.float64, device="cuda", generator=g)
    # rows of very different size: the row scaling must keep small rows accurate
    At *= torch.logspace(-6, 3, m, dtype=torch.float64, device="cuda")[None, :]
    Bt *= torch.logspace(2, -4, n, dtype=torch.float64, device="cuda")[None, :]
    Ct = torch.randn(n, m, dtype=torch.float64, device="cuda", generator=g)
    ref = 0.75 * (At.T @ Bt) - 0.5 * Ct.T
    _split_gemm(gpu_lib, At, Bt, Ct, 0.75, -0.5)
    got = Ct.T
    bound = 1e-13 * k * At.abs().amax(dim=0)[:, None] * Bt.abs().amax(dim=0)[None, :] + 1e-15 * ref.abs()
    assert bool(((got - ref).abs() <= bound).all()), float(((got - ref).abs() / bound).max())


def test_mixed_ao_to_mo_matches_fp64(gpu_lib):
    """GCI_PREC_MIXED on one decomposition: Rkab and the MO integrals it reconstructs
    agree with the FP64 transform to 1e-8 (the bound of the FP64 oracle parity)."""
    mol = molecules.config("c1")
    tb, ob = both(mol)
    res = cg.chol_gammcor_Rkpq(tb, cg.CHOL_ACCURACY_TIGHT, materialize=False)
    nocc, nvirt, seed = molecules.MO_SPLIT["c1"]
    Cm = molecules.mo_coefficients(tb.NAO, seed)
    ref = cg.chol_gammcor_Rkab(Cm, 1, nocc, Cm, nocc + 1, nocc + nvirt, 1024, res, tb)
    got = cg.chol_gammcor_Rkab(Cm, 1, nocc, Cm, nocc + 1, nocc + nvirt, 1024, res, tb, precision="mixed")
    assert np.max(np.abs(got - ref)) < 1e-8
    assert np.max(np.abs(got.T @ got - ref.T @ ref)) < 1e-8


def test_mixed_step1_gives_an_equivalent_decomposition(gpu_lib):
    """GCI_FLAG_MIXED_STEP1: the split-precision M - L L^T only steers the pivot
    search (the vectors are rebuilt in FP64 in step 2).  The pivot sequence matches
    the FP64 search at shell-pair level, and step 2 on its pivots agrees with the
    oracle to 1e-8."""
    mol = molecules.small_molecule(21, natoms=3, recipe=molecules.RECIPE_C1, nprim=(3, 4))
    tb, ob = both(mol)
    ref = cg.chol_gammcor_Rkpq(tb, cg.CHOL_ACCURACY_TIGHT)
    got = cg.chol_gammcor_Rkpq(tb, cg.CHOL_ACCURACY_TIGHT, mixed_step1=True)
    assert got.Chol2Data.NVecs == ref.Chol2Data.NVecs
    ch = O.cholesky(ob, mol.tau)
    owner = np.zeros(ch.norbpairs, dtype=np.int64)
    for sp in range(ch.nshellpairs):
        owner[ch.shellpairloc[sp, 0]:ch.shellpairloc[sp, 0] + ch.shellpairdim[sp]] = sp
    np.testing.assert_array_equal(owner[got.pivot_order - 1], owner[ref.pivot_order - 1])
    chf = O.cholesky(ob, mol.tau, forced_order=got.pivot_order - 1)
    from helpers import vectors_full_order
    Rg = vectors_full_order(got.Rkpq, got.Chol2Data.ShellPairLoc, got.Chol2Data.ShellPairDim)
    Ro = O.full_order_vectors(chf)
    assert np.max(np.abs(Rg.T @ Rg - Ro.T @ Ro)) < 1e-8
    O.free(ch)
    O.free(chf)
