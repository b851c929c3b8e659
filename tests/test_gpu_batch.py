"""GPU tests of gci_rkpq_batch: many independent molecules decomposed
concurrently (one CUDA stream per worker) give the same pivots and vectors as
one gci_rkpq call per molecule, and the batch agrees with the oracle on the
GPU's pivot set (reconstructed (pq|rs) within 1e-8, as the single-molecule
parity tests); a failing molecule fails the whole call with no handle out.

The molecules are the smallest of the 64-molecule c3 workload (c1 shell recipe,
l <= 2, 8 bohr cube, tau = 1e-5): one call mixes molecules of different size.
"""
import ctypes as C

import numpy as np
import pytest

from gammcor_integrals_b200 import _capi, basis, molecules
from gammcor_integrals_b200 import cholesky_gammcor as cg
from oracle import oracle as O

from helpers import vectors_full_order

pytestmark = pytest.mark.gpu


def _c3_small(n):
    counts = np.random.default_rng(3).integers(3, 31, 64)
    idx = sorted(range(64), key=lambda i: counts[i])[:n]
    return [molecules.config("c3", i) for i in idx]


def _vectors(v):
    d = v.Chol2Data
    return vectors_full_order(v.Rkpq, d.ShellPairLoc, d.ShellPairDim)


def test_batch_matches_single_calls(gpu_lib):
    mols = _c3_small(8)
    tbs = [basis.from_molecule(m) for m in mols]
    batch = cg.chol_gammcor_Rkpq_batch(tbs, cg.CHOL_ACCURACY_DEFAULT, nstreams=4)
    for tb, vb in zip(tbs, batch):
        vs = cg.chol_gammcor_Rkpq(tb, cg.CHOL_ACCURACY_DEFAULT)
        assert vb.Chol2Data.NVecs == vs.Chol2Data.NVecs
        np.testing.assert_array_equal(vb.pivot_order, vs.pivot_order)
        np.testing.assert_allclose(_vectors(vb), _vectors(vs), rtol=0, atol=1e-12)


def test_batch_against_oracle(gpu_lib):
    mols = _c3_small(3)
    tbs = [basis.from_molecule(m) for m in mols]
    batch = cg.chol_gammcor_Rkpq_batch(tbs, cg.CHOL_ACCURACY_DEFAULT, nstreams=3)
    for m, v in zip(mols, batch):
        ob = O.make_basis(m.atoms, m.shells)
        # step 2 of the oracle on the batch's pivot sequence: the same vectors up to rounding
        ch = O.cholesky(ob, m.tau, forced_order=v.pivot_order - 1)
        R = _vectors(v)
        Ro = O.full_order_vectors(ch)
        O.free(ch)
        assert np.max(np.abs(R.T @ R - Ro.T @ Ro)) < 1e-8


def test_batch_error_returns_no_handles(gpu_lib):
    mols = _c3_small(3)
    tbs = [basis.from_molecule(m) for m in mols]
    views = [tb.c_struct() for tb in tbs]
    views[1].nshellparams = 0          # an empty basis: rejected by the host set-up of molecule 1
    arr = (_capi.gci_basis * 3)(*views)
    hs = (C.c_void_p * 3)()
    rc = gpu_lib.gci_rkpq_batch(3, arr, 1, 0.0, 0, 2, hs)
    assert rc == -1                    # GCI_ERR_ARG
    assert all(h is None for h in hs)
    assert b"molecule 1" in gpu_lib.gci_last_error()
