"""GPU parity tests: libgci.so (through the C ABI) against the CPU oracle.

Tolerances: Boys 1e-13 relative (same table scheme); ERIs 1e-12 relative to
the largest integral (same two-centre Hermite form, different summation order);
reconstructed (pq|rs) = sum_k R_kpq R_krs and MO integrals within 1e-8
absolute of the oracle's own reconstructions; identical pivot sequences.
"""
import numpy as np
import pytest

from gammcor_integrals_b200 import _capi
from gammcor_integrals_b200 import cholesky_gammcor as cg
from gammcor_integrals_b200 import molecules
from oracle import oracle as O

from helpers import both, full_order_pairs, vectors_full_order

pytestmark = pytest.mark.gpu


def test_boys_matches_oracle(gpu_lib):
    rng = np.random.default_rng(0)
    x = np.concatenate([[0.0, 1e-12, 0.05, 24.999999, 25.0, 25.000001, 80.0],
                        rng.uniform(0, 30, 2000), rng.uniform(0, 1, 200)])
    for m in (0, 1, 4, 8, 12, 20):
        out = np.zeros((x.size, m + 1))
        _capi.check(gpu_lib.gci_boys(m, x.size, _capi.ptr(x), _capi.ptr(out)))
        ref = O.boys(m, x)
        assert np.max(np.abs(out - ref) / np.abs(ref)) < 1e-13


def _eri_pairs_gpu(tb):
    nao = tb.NAO
    npq = nao * (nao + 1) // 2
    out = np.zeros((npq, npq), order="F")
    s = tb.c_struct()
    import ctypes as C
    _capi.check(_capi.lib().gci_eri_pairs(C.byref(s), 0.0, _capi.ptr(out), npq))
    return out


def _vdiag_order_pairs(ob):
    pairs = []
    ns = len(ob.L)
    for B in range(ns):
        for A in range(B, ns):
            Na, Nb = 2 * int(ob.L[A]) + 1, 2 * int(ob.L[B]) + 1
            for b in range(Nb):
                for a in range(b if A == B else 0, Na):
                    pairs.append((ob.shell_loc[A] + a, ob.shell_loc[B] + b))
    return np.array(pairs)


class _Variants:
    """Force one kernel family on the product stages: "hermite" (the Hermite-matrix
    kernels) or a class-kernel variant 0..3 on every class that has it (-1 keeps
    the current variants); restore everything on exit."""

    def __init__(self, lib, variant):
        self.lib, self.variant, self.saved, self.hm = lib, variant, {}, None

    def __enter__(self):
        self.hm = self.lib.gci_eri_hm(1 if self.variant == "hermite" else 0)
        if self.variant != "hermite":
            for tb in range(10):
                for tk in range(tb + 1):
                    self.saved[(tb, tk)] = self.lib.gci_eri_variant(tb, tk, -1)
                    self.lib.gci_eri_variant(tb, tk, self.variant)   # GCI_ERR_ARG where not built
        return self

    def __exit__(self, *exc):
        for (tb, tk), v in self.saved.items():
            self.lib.gci_eri_variant(tb, tk, v)
        self.lib.gci_eri_hm(self.hm)


@pytest.mark.parametrize("variant", ["hermite", 0, 1, 2, 3])
@pytest.mark.parametrize("recipe,seed,natoms", [(molecules.RECIPE_C1, 11, 3), (molecules.RECIPE_C2, 12, 2)])
def test_eri_blocks_all_classes(gpu_lib, recipe, seed, natoms, variant):
    mol = molecules.small_molecule(seed, natoms=natoms, recipe=recipe, nprim=(3, 4))
    tb, ob = both(mol)
    with _Variants(gpu_lib, variant):
        V = _eri_pairs_gpu(tb)
    G = O.eri_full(ob)
    pq = _vdiag_order_pairs(ob)
    ref = G[pq[:, 0], pq[:, 1]][:, pq[:, 0], pq[:, 1]]
    err = np.max(np.abs(V - ref))
    # two-centre Hermite form in both: agreement to rounding of the largest integral
    assert err < 1e-12 * max(1.0, np.max(np.abs(ref))), err


def test_autotune_keeps_results(gpu_lib):
    mol = molecules.small_molecule(12, natoms=2, recipe=molecules.RECIPE_C2, nprim=(3, 4))
    tb, ob = both(mol)
    secs = np.zeros(400)
    s = tb.c_struct()
    import ctypes as C
    # the tuner's choice is process-wide: restore the defaults afterwards so that the
    # other tests do not depend on the order in which they run
    with _Variants(gpu_lib, -1):
        _capi.check(gpu_lib.gci_autotune_eri(C.byref(s), 64, _capi.ptr(secs)))
        assert np.all(secs >= 0) and np.count_nonzero(secs) > 0
        V = _eri_pairs_gpu(tb)
    G = O.eri_full(ob)
    pq = _vdiag_order_pairs(ob)
    ref = G[pq[:, 0], pq[:, 1]][:, pq[:, 0], pq[:, 1]]
    assert np.max(np.abs(V - ref)) < 1e-12 * max(1.0, np.max(np.abs(ref)))


def _shellpair_of_full(ch):
    """FULL orbital-pair index -> BASE shell pair index."""
    owner = np.zeros(ch.norbpairs, dtype=np.int64)
    for sp in range(ch.nshellpairs):
        f = ch.shellpairloc[sp, 0]
        owner[f:f + ch.shellpairdim[sp]] = sp
    return owner


def _exact_full_order(ob, ch):
    G = O.eri_full(ob)
    pq = full_order_pairs(ch.nshellpairs, ch.shellpairs, ob)
    return G[pq[:, 0], pq[:, 1]][:, pq[:, 0], pq[:, 1]]


def _run_both(mol, decode_storage=False):
    tb, ob = both(mol)
    res = cg.chol_gammcor_Rkpq(tb, cg.CHOL_ACCURACY_TIGHT, decode_storage=decode_storage)
    ch = O.cholesky(ob, mol.tau, decode_storage=decode_storage)
    c2 = res.Chol2Data
    assert c2.NOrbPairs == ch.norbpairs
    assert c2.NShellPairs == ch.nshellpairs
    np.testing.assert_array_equal(c2.ShellPairs.T - 1, ch.shellpairs)
    np.testing.assert_array_equal(c2.ShellPairLoc.T - 1, ch.shellpairloc)
    np.testing.assert_array_equal(c2.SubsetDim, ch.subsetdim)
    return tb, ob, res, ch


def _assert_step2_parity(tb, ob, res, mol, decode_storage=False):
    """Step 2 + full-dimension vectors on the GPU's own pivot set agree with the
    oracle to 1e-8 (independent of how symmetry ties were broken in step 1)."""
    c2 = res.Chol2Data
    ch = O.cholesky(ob, mol.tau, decode_storage=decode_storage, forced_order=res.pivot_order - 1)
    np.testing.assert_array_equal(c2.Pivots, ch.pivots)
    np.testing.assert_array_equal(c2.PivotOrbPairs - 1, ch.pivorbpairs)
    np.testing.assert_array_equal(c2.PivotShellPairLoc - 1, ch.pivshellpairloc)
    Rg = vectors_full_order(res.Rkpq, c2.ShellPairLoc, c2.ShellPairDim)
    Ro = O.full_order_vectors(ch)
    assert np.max(np.abs(Rg.T @ Rg - Ro.T @ Ro)) < 1e-8
    # Inv_L inherits the conditioning of V_JJ (its smallest pivots are ~ tau, and
    # the reference's folded decode of diagonal-shell-pair pivots can pick nearly
    # dependent columns), so elementwise agreement is only required loosely; the
    # vectors it produces are compared through R^T R above.
    assert np.max(np.abs(c2.Inv_L - ch.inv_l)) < 1e-2 * np.max(np.abs(ch.inv_l))
    return ch


def test_cholesky_strict_nondegenerate(gpu_lib):
    """s shells only: no symmetry-equivalent diagonals, so the pivot sequence,
    the pivot set, Inv_L and the vectors must all match."""
    mol = molecules.small_molecule(41, natoms=4, recipe=(0, 0, 0, 0), nprim=(3, 4))
    tb, ob, res, ch = _run_both(mol)
    c2 = res.Chol2Data
    assert c2.NVecs == ch.nvecs
    np.testing.assert_array_equal(res.pivot_order - 1, ch.pivot_order)
    np.testing.assert_allclose(res.pivot_dmax, ch.pivot_dmax, rtol=0, atol=1e-12 * ch.pivot_dmax.max())
    np.testing.assert_array_equal(c2.Pivots, ch.pivots)
    Rg = vectors_full_order(res.Rkpq, c2.ShellPairLoc, c2.ShellPairDim)
    Ro = O.full_order_vectors(ch)
    assert np.max(np.abs(Rg.T @ Rg - Ro.T @ Ro)) < 1e-8
    assert np.max(np.abs(c2.Inv_L - ch.inv_l)) < 1e-6 * np.max(np.abs(ch.inv_l))


def _assert_equivalent_sequences(res, ch):
    """Pivot sequences agree up to symmetry ties: the same count, the same shell
    pair at every step, and identical selections with matching residual
    diagonals up to the first tie (components of one shell pair whose
    diagonals are equal by symmetry, so rounding decides the winner)."""
    assert res.Chol2Data.NVecs == ch.nvecs
    owner = _shellpair_of_full(ch)
    g, o = res.pivot_order - 1, ch.pivot_order
    np.testing.assert_array_equal(owner[g], owner[o])
    diff = np.nonzero(g != o)[0]
    first = diff[0] if diff.size else g.size
    atol = 1e-12 * ch.pivot_dmax.max()
    np.testing.assert_allclose(res.pivot_dmax[:first + 1], ch.pivot_dmax[:first + 1], rtol=0, atol=atol)


@pytest.mark.parametrize("recipe,seed,natoms", [(molecules.RECIPE_C1, 21, 3), (molecules.RECIPE_C2, 22, 2)])
def test_cholesky_pivots_and_vectors(gpu_lib, recipe, seed, natoms):
    mol = molecules.small_molecule(seed, natoms=natoms, recipe=recipe, nprim=(3, 4))
    tb, ob, res, ch = _run_both(mol)
    _assert_equivalent_sequences(res, ch)
    # both decompositions reproduce the exact integrals to within tau
    V = _exact_full_order(ob, ch)
    Rg = vectors_full_order(res.Rkpq, res.Chol2Data.ShellPairLoc, res.Chol2Data.ShellPairDim)
    assert np.max(np.abs(V - Rg.T @ Rg)) <= 1.001 * mol.tau
    _assert_step2_parity(tb, ob, res, mol)


def test_cholesky_storage_decode(gpu_lib):
    mol = molecules.small_molecule(23, natoms=3)
    tb, ob, res, ch = _run_both(mol, decode_storage=True)
    _assert_equivalent_sequences(res, ch)
    _assert_step2_parity(tb, ob, res, mol, decode_storage=True)


def test_rkab_direct_and_materialised(gpu_lib):
    mol = molecules.small_molecule(31, natoms=3)
    tb, ob = both(mol)
    res = cg.chol_gammcor_Rkpq(tb, cg.CHOL_ACCURACY_TIGHT)
    ch = _assert_step2_parity(tb, ob, res, mol)
    nao = tb.NAO
    Cm = molecules.mo_coefficients(nao, 7)
    a0, a1, b0, b1 = 1, 6, 7, nao
    ref = O.mo_transf(ch, ob, Cm, a0 - 1, a1 - 1, Cm, b0 - 1, b1 - 1)
    got = cg.chol_gammcor_Rkab(Cm, a0, a1, Cm, b0, b1, 256, res, tb)
    assert np.max(np.abs(got - ref)) < 1e-8
    assert np.max(np.abs(got.T @ got - ref.T @ ref)) < 1e-8
    res2 = cg.chol_gammcor_Rkpq(tb, cg.CHOL_ACCURACY_TIGHT, materialize=False)
    np.testing.assert_array_equal(res2.pivot_order, res.pivot_order)
    got2 = cg.chol_gammcor_Rkab(Cm, a0, a1, Cm, b0, b1, 1, res2, tb)
    assert np.max(np.abs(got2 - ref)) < 1e-8


def test_c1_job_parity(gpu_lib):
    """The c1 benchmark configuration end to end (10 atoms, NAO = 140, tau = 1e-6,
    MO 20 occupied x 60 virtual of the seeded C) against the oracle: the pivot
    sequence at shell-pair level with residual diagonals up to the first symmetry
    tie; on the GPU's pivot set the vectors through R^T R, V_JJ's inverse factor
    Inv_L, and Rkab with the MO integrals it reconstructs, through the stored and
    the direct AO->MO paths, all to 1e-8 absolute."""
    mol = molecules.config("c1")
    tb, ob, res, ch = _run_both(mol)
    _assert_equivalent_sequences(res, ch)
    ch2 = _assert_step2_parity(tb, ob, res, mol)
    # Inv_L elementwise, relative to its largest entry (~1/sqrt(tau)): the pivot block's
    # condition number (max diagonal / tau ~ 1e7) times FP64 rounding; measured 2.4e-9
    rel = np.max(np.abs(res.Chol2Data.Inv_L - ch2.inv_l)) / np.max(np.abs(ch2.inv_l))
    assert rel < 1e-7, rel
    nocc, nvirt, seed = molecules.MO_SPLIT["c1"]
    Cm = molecules.mo_coefficients(tb.NAO, seed)
    ref = O.mo_transf(ch2, ob, Cm, 0, nocc - 1, Cm, nocc, nocc + nvirt - 1)
    got = cg.chol_gammcor_Rkab(Cm, 1, nocc, Cm, nocc + 1, nocc + nvirt, 1024, res, tb)
    assert np.max(np.abs(got - ref)) < 1e-8
    assert np.max(np.abs(got.T @ got - ref.T @ ref)) < 1e-8
    res2 = cg.chol_gammcor_Rkpq(tb, cg.CHOL_ACCURACY_TIGHT, materialize=False)
    np.testing.assert_array_equal(res2.pivot_order, res.pivot_order)
    got2 = cg.chol_gammcor_Rkab(Cm, 1, nocc, Cm, nocc + 1, nocc + nvirt, 1024, res2, tb)
    assert np.max(np.abs(got2 - ref)) < 1e-8
    O.free(ch)
    O.free(ch2)


def test_rkab_out_of_core_matches(gpu_lib, monkeypatch):
    """The direct AO->MO path with Vab staged in the caller's host array and Inv_L applied
    block by block from there (used when the host output does not fit on the device;
    forced here by GCI_RKAB_OUT_OF_CORE) gives the in-core result; an 8 MB buffer splits
    the full-dimension integrals into several pivot chunks."""
    mol = molecules.config("c1")
    tb, _ = both(mol)
    res = cg.chol_gammcor_Rkpq(tb, cg.CHOL_ACCURACY_TIGHT, materialize=False)
    nocc, nvirt, seed = molecules.MO_SPLIT["c1"]
    Cm = molecules.mo_coefficients(tb.NAO, seed)
    ref = cg.chol_gammcor_Rkab(Cm, 1, nocc, Cm, nocc + 1, nocc + nvirt, 1024, res, tb)
    monkeypatch.setenv("GCI_RKAB_OUT_OF_CORE", "1")
    got = cg.chol_gammcor_Rkab(Cm, 1, nocc, Cm, nocc + 1, nocc + nvirt, 8, res, tb)
    assert np.max(np.abs(got - ref)) < 1e-11
