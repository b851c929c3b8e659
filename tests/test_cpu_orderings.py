"""AO orderings of external programs against expectations written out by hand
from the position tables of Auto2eInterface.f90 (MOLPRO_* :41-59, ORCA_* :25-39,
DALTON_*/PYSCF_* :61-92, OPEN_MOLCAS_* :94-142 with the within-atom example of
:95-127, MOLPRO_CART_* :144-213) and the ORCA phase rule of
auto2e_interface_ApplyOrcaPhases_Vector (:517-566): f shells flip m = +-3,
g and h shells m = +-3 and +-4 (not m = +-5 of h).

Map_extao2ao(p) is the Auto2e position (1-based) of external position p."""
import numpy as np
import pytest

from gammcor_integrals_b200 import auto2e_interface as ai, basis as gbasis
from gammcor_integrals_b200.molecules import Molecule


def _basis(shell_ls, spher=True, natoms=1):
    """One primitive per shell; shells listed per atom in `shell_ls` (same on every atom)."""
    atoms = [[0.0, 0.0, 1.5 * a] for a in range(natoms)]
    shells = [(a, L, np.array([1.0]), np.array([1.0])) for a in range(natoms) for L in shell_ls]
    return gbasis.from_molecule(Molecule(atoms=atoms, shells=shells, tau=1e-6, name="ord"), spher=spher)


# one atom with s, p, d, f shells: spherical positions s 1, p 2-4, d 5-9, f 10-16
SPDF_EXPECTED = {
    # d: d0 d2- d1+ d2+ d1- ; f: f1+ f1- f0 f3+ f2- f3- f2+
    ai.ORBITAL_ORDERING_MOLPRO: [1, 2, 3, 4, 7, 5, 8, 9, 6, 14, 12, 13, 16, 11, 10, 15],
    # p: pz px py ; d: d0 d1+ d1- d2+ d2- ; f: f0 f1+ f1- f2+ f2- f3+ f3-
    ai.ORBITAL_ORDERING_ORCA: [1, 4, 2, 3, 7, 8, 6, 9, 5, 13, 14, 12, 15, 11, 16, 10],
    # m = -L..L: the Auto2e order itself
    ai.ORBITAL_ORDERING_DALTON: list(range(1, 17)),
    ai.ORBITAL_ORDERING_PYSCF: list(range(1, 17)),
}


@pytest.mark.parametrize("ordering", sorted(SPDF_EXPECTED))
def test_spherical_spdf_maps(ordering):
    tb = _basis((0, 1, 2, 3))
    assert tb.NAO == 16
    m_ext, m_ao = ai.auto2e_interface_AOMap(tb, ordering)
    assert list(m_ext) == SPDF_EXPECTED[ordering]
    assert all(m_ao[m_ext[p] - 1] == p + 1 for p in range(16))


def test_spherical_g_h_maps():
    tb = _basis((4, 5))   # g at 1-9, h at 10-20
    m_ext, _ = ai.auto2e_interface_AOMap(tb, ai.ORBITAL_ORDERING_MOLPRO)
    # g: g0 g2- g1+ g4+ g1- g2+ g4- g3+ g3- ; h: h1+ h1- h2+ h3+ h4- h3- h4+ h5- h0 h5+ h2-
    assert list(m_ext) == [5, 3, 6, 9, 4, 7, 1, 8, 2] + [9 + p for p in (7, 5, 8, 9, 2, 3, 10, 1, 6, 11, 4)]
    m_ext, _ = ai.auto2e_interface_AOMap(tb, ai.ORBITAL_ORDERING_ORCA)
    # g0 g1+ g1- g2+ g2- g3+ g3- g4+ g4- ; h0 h1+ h1- ... h5+ h5-
    assert list(m_ext) == [5, 6, 4, 7, 3, 8, 2, 9, 1] + [9 + p for p in (6, 7, 5, 8, 4, 9, 3, 10, 2, 11, 1)]


def test_open_molcas_within_atom_order():
    # the reference's example atom: shells s, p, p, d, d, s at 1, 2-4, 5-7, 8-12, 13-17, 18
    tb = _basis((0, 1, 1, 2, 2, 0), natoms=2)
    m_ext, _ = ai.auto2e_interface_AOMap(tb, ai.ORBITAL_ORDERING_OPEN_MOLCAS)
    atom = [1, 18,                      # s (shell 1), s (shell 6)
            2, 5, 3, 6, 4, 7,           # px, py, pz of shells 2 and 3
            8, 13, 9, 14, 10, 15, 11, 16, 12, 17]   # d-2 .. d+2 of shells 4 and 5
    assert list(m_ext) == atom + [18 + p for p in atom]


def test_cartesian_molpro_map():
    tb = _basis((0, 1, 2, 3), spher=False)
    assert tb.NAO == 20
    m_ext, _ = ai.auto2e_interface_AOMap(tb, ai.ORBITAL_ORDERING_MOLPRO)
    # d: xx yy zz xy xz yz ; f: xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz
    assert list(m_ext) == [1, 2, 3, 4, 5, 8, 10, 6, 7, 9, 11, 17, 20, 12, 13, 14, 18, 16, 19, 15]
    with pytest.raises(ValueError):
        ai.auto2e_interface_AOMap(tb, ai.ORBITAL_ORDERING_ORCA)


@pytest.mark.parametrize("shell_ls,flipped", [((0, 1, 2, 3), [10, 16]),
                                              ((4,), [1, 2, 8, 9]),
                                              ((5,), [2, 3, 9, 10]),
                                              ((3, 4), [1, 7, 8, 9, 15, 16])])
def test_orca_phases(shell_ls, flipped):
    tb = _basis(shell_ls)
    n = tb.NAO
    sign = np.ones(n)
    sign[np.array(flipped) - 1] = -1.0
    X = np.random.default_rng(0).normal(size=(n, n + 3))
    Y = ai.auto2e_interface_ApplyOrcaPhases_Matrix(X, tb, False)
    ref = X.copy()
    ref[:, :n] *= sign[:, None]
    np.testing.assert_array_equal(Y, ref)
    Z = ai.auto2e_interface_ApplyOrcaPhases_Matrix(X[:, :n], tb, True)
    np.testing.assert_array_equal(Z, X[:, :n] * sign[:, None] * sign[None, :])


def test_transform_uses_map_direction():
    """AngFuncTransf from the external order places external row p at Auto2e row Map_extao2ao(p)."""
    tb = _basis((0, 1, 2, 3))
    X = np.arange(16, dtype=float)[:, None] + 1.0   # external row p holds p + 1
    Y = ai.auto2e_interface_AngFuncTransf(X, True, False, tb, ai.ORBITAL_ORDERING_ORCA)
    for p, q in enumerate(SPDF_EXPECTED[ai.ORBITAL_ORDERING_ORCA]):
        assert Y[q - 1, 0] == p + 1
