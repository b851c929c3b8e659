"""GPU tests of the adjoint path (gci_coulomb_grad*): the Coulomb energy
J = 1/2 sum D_pq (pq|rs) D_rs, its nuclear gradient and the Coulomb matrix
against the CPU oracle (orc_coulomb_energy_grad: derivative integrals from
shells raised and lowered by one unit of angular momentum, an independent
route), central finite differences of the GPU energy, and the
torch.autograd.Function.

Tolerances: energy 1e-11 relative; gradient and Coulomb matrix 1e-9 of their
largest element (FP64 throughout, different summation order); finite
differences (h = 1e-4 bohr) 1e-6 absolute.
"""
import numpy as np
import pytest

from gammcor_integrals_b200 import coulomb_grad as cgr
from gammcor_integrals_b200 import molecules
from oracle import oracle as O

from helpers import both

pytestmark = pytest.mark.gpu


def _density(nao, seed, rank=6, scale=0.1):
    X = np.random.default_rng(seed).normal(0.0, scale, (nao, rank))
    return X @ X.T


@pytest.mark.parametrize("recipe,seed,natoms,omega", [
    ((0, 1, 2), 21, 3, 0.0),
    ((0, 0, 1, 2), 22, 2, 0.0),
    ((1, 2, 3), 23, 2, 0.0),
    ((0, 1, 2), 24, 2, 0.7),
])
def test_energy_and_gradient_match_oracle(gpu_lib, recipe, seed, natoms, omega):
    mol = molecules.small_molecule(seed, natoms=natoms, recipe=recipe, cube=4.0)
    tb, ob = both(mol)
    D = _density(tb.NAO, seed)
    e, g, _ = cgr.coulomb_energy_grad(tb, D, omega=omega)
    kappa = 1.0 / omega ** 2 if omega > 0 else 0.0
    e_ref, g_ref = O.coulomb_energy_grad(ob, D, kappa=kappa)
    assert abs(e - e_ref) <= 1e-11 * abs(e_ref)
    assert np.max(np.abs(g - g_ref)) <= 1e-9 * max(1.0, np.max(np.abs(g_ref)))
    assert np.max(np.abs(g.sum(axis=0))) <= 1e-9 * max(1.0, np.max(np.abs(g_ref)))


def test_coulomb_matrix_matches_eri_contraction(gpu_lib):
    mol = molecules.small_molecule(31, natoms=2, recipe=(0, 1, 2, 3), cube=4.0)
    tb, ob = both(mol)
    rng = np.random.default_rng(31)
    D = rng.normal(size=(tb.NAO, tb.NAO))      # not symmetric: the library symmetrises it
    e, _, jm = cgr.coulomb_energy_grad(tb, D, want_jmat=True)
    eri = O.eri_full(ob)
    Ds = 0.5 * (D + D.T)
    jref = np.einsum("pqrs,rs->pq", eri, Ds)
    assert np.max(np.abs(jm - jref)) <= 1e-9 * np.max(np.abs(jref))
    assert abs(e - 0.5 * np.sum(Ds * jref)) <= 1e-11 * abs(e)


def test_c4_gradient_matches_finite_differences(gpu_lib):
    """The c4 workload (20 atoms, 280 AOs, D = X X^T, X ~ N(0, 0.1^2) of 280 x 30):
    central differences with h = 1e-4 bohr on three atoms."""
    mol = molecules.config("c4")
    tb, _ = both(mol)
    D = _density(tb.NAO, 104, rank=30)
    _, g, _ = cgr.coulomb_energy_grad(tb, D)
    h = 1e-4
    coords = mol.atoms
    for at in (0, 7, 19):
        for ax in range(3):
            cp, cm = coords.copy(), coords.copy()
            cp[at, ax] += h
            cm[at, ax] -= h
            ep = cgr.coulomb_energy_grad(cgr.with_coords(tb, cp), D)[0]
            em = cgr.coulomb_energy_grad(cgr.with_coords(tb, cm), D)[0]
            assert abs((ep - em) / (2 * h) - g[at, ax]) <= 1e-6, (at, ax)
    assert np.max(np.abs(g.sum(axis=0))) <= 1e-8 * np.max(np.abs(g))


def test_autograd_function(gpu_lib):
    import torch
    mol = molecules.small_molecule(41, natoms=3, recipe=(0, 1, 2), cube=4.0)
    tb, _ = both(mol)
    D = _density(tb.NAO, 41)
    e, g, jm = cgr.coulomb_energy_grad(tb, D, want_jmat=True)
    coords = torch.tensor(mol.atoms, dtype=torch.float64, device="cuda", requires_grad=True)
    Dt = torch.tensor(D, dtype=torch.float64, device="cuda", requires_grad=True)
    J = cgr.coulomb_energy(coords, Dt, tb)
    (2.5 * J).backward()
    assert abs(J.item() - e) <= 1e-12 * abs(e)
    np.testing.assert_allclose(coords.grad.cpu().numpy(), 2.5 * g, rtol=0, atol=1e-12 * np.max(np.abs(g)))
    np.testing.assert_allclose(Dt.grad.cpu().numpy(), 2.5 * jm, rtol=0, atol=1e-12 * np.max(np.abs(jm)))
