"""CPU tests of the C ABI library: it loads without a GPU, exports every
entry point of include/gci.h, and its host-only numerics agree with the
oracle (normalisation, solid-harmonic coefficients)."""
import re
from pathlib import Path

import numpy as np
import pytest

from gammcor_integrals_b200 import _capi, basis as gbasis, molecules
from oracle import oracle as O

ROOT = Path(__file__).resolve().parent.parent


def test_library_exports_header_symbols():
    L = _capi.lib()
    header = (ROOT / "include" / "gci.h").read_text()
    declared = set(re.findall(r"\b(gci_[a-z0-9_]+)\s*\(", header))
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(L, name), name
    assert declared == set(_capi.EXPORTS)


def test_spher_coeffs_match_oracle():
    for L in range(0, 6):
        U = np.zeros((2 * L + 1, (L + 1) * (L + 2) // 2))
        _capi.check(_capi.lib().gci_spher_coeffs(L, _capi.ptr(U)))
        np.testing.assert_allclose(U, O.spher_u(L), rtol=1e-13, atol=1e-15)


def test_normalisation_matches_oracle():
    mol = molecules.small_molecule(5, natoms=2, recipe=molecules.RECIPE_C2, nprim=(3, 6))
    tb = gbasis.from_molecule(mol)
    ob = O.make_basis(mol.atoms, mol.shells)
    for s in range(tb.NShells):
        np.testing.assert_allclose(tb.CntrCoeffs[:tb.NPrimitives[s], s],
                                   ob.coefs[ob.prim_off[s]:ob.prim_off[s] + ob.nprim[s]], rtol=1e-13)
    assert tb.NAOSpher == ob.nao


def test_noalloc_rejects_oversized_basis_before_device_work():
    # 8 f shells of 40 primitives on one centre need ~42 MB of pair records,
    # beyond the fixed scratch; the size check comes before any CUDA call, so
    # this runs without a GPU (the output pointer is never dereferenced)
    import ctypes as C
    import torch
    if torch.cuda.is_available():
        # with a device the library could reach the output pointer; the GPU test
        # test_zz_no_alloc.py covers the rejection with a real buffer
        pytest.skip("host-only check of the size limit; a CUDA device is visible")
    mol = molecules.random_molecule(77, 1, 4.0, (3,) * 8, (40, 40), (0.1, 1e3))
    tb = gbasis.from_molecule(mol)
    s = tb.c_struct()
    npq = tb.NAO * (tb.NAO + 1) // 2
    rc = _capi.lib().gci_eri_pairs_noalloc(C.byref(s), 0.0, C.c_void_p(256), npq, None)
    assert rc == _capi.GCI_ERR_BUFFER
    msg = _capi.lib().gci_last_error().decode()
    assert "scratch" in msg and str(_capi.GCI_NOALLOC_SCRATCH_BYTES) in msg


def test_coulomb_grad_and_batch_argument_errors_without_device_work():
    """Argument checks of the adjoint and batch entry points come before any
    CUDA call (no GPU needed): a NULL density, nothing requested, and an empty
    batch."""
    import ctypes as C
    mol = molecules.small_molecule(3, natoms=2, recipe=(0, 1))
    tb = gbasis.from_molecule(mol)
    s = tb.c_struct()
    L = _capi.lib()
    e = C.c_double()
    g = np.zeros(3 * tb.NAtoms)
    assert L.gci_coulomb_grad(C.byref(s), 0.0, None, tb.NAO, C.byref(e), _capi.ptr(g), None, tb.NAO) == -1
    assert b"D is NULL" in L.gci_last_error()
    D = np.eye(tb.NAO)
    assert L.gci_coulomb_grad(C.byref(s), 0.0, _capi.ptr(D), tb.NAO, None, None, None, tb.NAO) == -1
    assert b"nothing requested" in L.gci_last_error()
    hs = (C.c_void_p * 1)()
    arr = (_capi.gci_basis * 1)(s)
    assert L.gci_rkpq_batch(0, arr, 1, 0.0, 0, 4, hs) == 0
    assert L.gci_rkpq_batch(-1, arr, 1, 0.0, 0, 4, hs) == -1


def test_adjoint_work_model():
    """flops.grad_class_flops counts the potential kernel's arithmetic: the
    contraction H(L1+1) H(L2) FMAs dominates, the recursion grows with N."""
    from gammcor_integrals_b200 import flops
    f = flops.grad_class_flops
    assert f(0, 0) == 30 + 3 * 1 + 25 + 3 * (flops.herm_n(1) - 1) + 2 * 4 * 1
    assert f(4, 4) > f(4, 3) > f(3, 3)
    w = np.zeros(49)
    w[2 * 7 + 1] = 10.0
    assert flops.grad_flops(w) == 10.0 * f(2, 1)


def test_split_gemm_argument_checks_without_device_work():
    """gci_dgemm_split validates its dimensions before any CUDA call (no GPU needed):
    negative sizes and leading dimensions below the row counts are GCI_ERR_ARG."""
    L = _capi.lib()
    assert L.gci_dgemm_split(-1, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4) == -1
    assert L.gci_dgemm_split(8, 4, 4, 1.0, None, 7, None, 4, 0.0, None, 8) == -1
    assert L.gci_dgemm_split(8, 4, 4, 1.0, None, 8, None, 3, 0.0, None, 8) == -1
    assert L.gci_dgemm_split(8, 4, 4, 1.0, None, 8, None, 4, 0.0, None, 8) == -1   # NULL operands
    assert b"NULL" in L.gci_last_error()
