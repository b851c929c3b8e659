"""TAOBasis and the basis set-up routines of the reference the path reads.

Mirrors src/basis/basis_definitions.f90:94-192 (TAOBasis), basis_Init_2
(src/basis/basis_sets.f90:659-824), basis_NormalizeCntrCoeffs (:894-945),
basis_CountOrbitals (:826-856) and SpherGTO_NormFactors
(src/basis/sphergto.f90:166-211).  Index arrays are 1-based, as the Fortran
type holds them; 2-D arrays are Fortran-ordered.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _capi


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


@dataclass
class TAOBasis:
    AtomCoords: np.ndarray          # (3, NAtoms)
    ShellCenters: np.ndarray        # (NShells,) 1-based
    ShellParamsIdx: np.ndarray      # (NShells,) 1-based
    ShellMomentum: np.ndarray       # (NShellParams,)
    NPrimitives: np.ndarray         # (NShellParams,)
    CntrCoeffs: np.ndarray          # (MaxNPrimitives, NShellParams), primitive norms folded in
    Exponents: np.ndarray           # (MaxNPrimitives, NShellParams)
    NormFactorsCart: np.ndarray     # (MaxNAngFuncCart, NShellParams)
    NormFactorsSpher: np.ndarray    # (MaxNAngFuncSpher, NShellParams)
    NAngFuncCart: np.ndarray
    NAngFuncSpher: np.ndarray
    ShellLocCart: np.ndarray        # 1-based
    ShellLocSpher: np.ndarray       # 1-based
    NAOCart: int
    NAOSpher: int
    LmaxGTO: int
    MaxNPrimitives: int
    SpherAO: bool = True

    @property
    def NAtoms(self) -> int:
        return self.AtomCoords.shape[1]

    @property
    def NShells(self) -> int:
        return self.ShellCenters.size

    @property
    def NShellParams(self) -> int:
        return self.ShellMomentum.size

    @property
    def NAO(self) -> int:
        return self.NAOSpher if self.SpherAO else self.NAOCart

    def c_struct(self):
        """gci_basis view of this basis (arrays are kept alive on the struct)."""
        nf = self.NormFactorsSpher if self.SpherAO else self.NormFactorsCart
        keep = [np.asfortranarray(self.AtomCoords, dtype=np.float64),
                np.ascontiguousarray(self.ShellCenters, dtype=np.int64),
                np.ascontiguousarray(self.ShellParamsIdx, dtype=np.int64),
                np.ascontiguousarray(self.ShellMomentum, dtype=np.int64),
                np.ascontiguousarray(self.NPrimitives, dtype=np.int64),
                np.asfortranarray(self.CntrCoeffs, dtype=np.float64),
                np.asfortranarray(self.Exponents, dtype=np.float64),
                np.asfortranarray(nf, dtype=np.float64)]
        s = _capi.gci_basis(self.NAtoms, self.NShells, self.NShellParams, self.CntrCoeffs.shape[0], nf.shape[0],
                            _capi.ptr(keep[0]), _capi.ptr(keep[1], _capi._pl), _capi.ptr(keep[2], _capi._pl),
                            _capi.ptr(keep[3], _capi._pl), _capi.ptr(keep[4], _capi._pl), _capi.ptr(keep[5]),
                            _capi.ptr(keep[6]), _capi.ptr(keep[7]), int(bool(self.SpherAO)))
        s._keep = keep
        return s


def basis_NormalizeCntrCoeffs(CntrCoeffs: np.ndarray, Exponents: np.ndarray, NPrimitives, ShellMomentum):
    """Rescale the contraction coefficients in place; return NormFactorsCart and NormFactorsSpher."""
    L = np.ascontiguousarray(ShellMomentum, dtype=np.int64)
    npr = np.ascontiguousarray(NPrimitives, dtype=np.int64)
    ldprim, nparams = CntrCoeffs.shape
    lmax = int(L.max())
    ncart_cart = np.zeros((ncart(lmax), nparams), order="F")
    ncart_sph = np.zeros((2 * lmax + 1, nparams), order="F")
    E = np.asfortranarray(Exponents, dtype=np.float64)
    assert CntrCoeffs.flags.f_contiguous and CntrCoeffs.dtype == np.float64
    _capi.check(_capi.lib().gci_normalize_basis(nparams, ldprim, _capi.ptr(L, _capi._pl), _capi.ptr(npr, _capi._pl),
                                                 _capi.ptr(E), _capi.ptr(CntrCoeffs), _capi.ptr(ncart_cart),
                                                 ncart_cart.shape[0], _capi.ptr(ncart_sph), ncart_sph.shape[0]))
    return ncart_cart, ncart_sph


def basis_CountOrbitals(ShellMomentum, ShellParamsIdx):
    L = np.asarray(ShellMomentum)
    nsph = 2 * L + 1
    ncar = (L + 1) * (L + 2) // 2
    per_shell_s = nsph[np.asarray(ShellParamsIdx) - 1]
    per_shell_c = ncar[np.asarray(ShellParamsIdx) - 1]
    locs = np.concatenate([[0], np.cumsum(per_shell_s)[:-1]]) + 1
    locc = np.concatenate([[0], np.cumsum(per_shell_c)[:-1]]) + 1
    return int(per_shell_s.sum()), int(per_shell_c.sum()), nsph, ncar, locs, locc


def basis_Init_2(AtomCoords, ShellCenters, ShellParamsIdx, ShellMomentum, NPrimitives, CntrCoeffs, Exponents,
                 NormFactorsCart, SpherAO: bool = True, NormFactorsSpher=None) -> TAOBasis:
    """basis_Init_2 (basis_sets.f90:659-824): CntrCoeffs are already normalised."""
    nsph_total, ncart_total, nsph, ncar, locs, locc = basis_CountOrbitals(ShellMomentum, ShellParamsIdx)
    if NormFactorsSpher is None:
        # SpherGTO_NormFactors is computed together with the coefficient
        # rescaling by basis_NormalizeCntrCoeffs in this package
        raise ValueError("pass NormFactorsSpher as returned by basis_NormalizeCntrCoeffs")
    return TAOBasis(AtomCoords=np.asfortranarray(AtomCoords, dtype=np.float64),
                    ShellCenters=np.asarray(ShellCenters, dtype=np.int64),
                    ShellParamsIdx=np.asarray(ShellParamsIdx, dtype=np.int64),
                    ShellMomentum=np.asarray(ShellMomentum, dtype=np.int64),
                    NPrimitives=np.asarray(NPrimitives, dtype=np.int64),
                    CntrCoeffs=np.asfortranarray(CntrCoeffs), Exponents=np.asfortranarray(Exponents),
                    NormFactorsCart=np.asfortranarray(NormFactorsCart),
                    NormFactorsSpher=np.asfortranarray(NormFactorsSpher),
                    NAngFuncCart=ncar, NAngFuncSpher=nsph, ShellLocCart=locc, ShellLocSpher=locs,
                    NAOCart=ncart_total, NAOSpher=nsph_total, LmaxGTO=int(np.max(ShellMomentum)),
                    MaxNPrimitives=int(np.max(NPrimitives)), SpherAO=SpherAO)


def from_molecule(mol, spher: bool = True) -> TAOBasis:
    """TAOBasis of a molecules.Molecule: one parameter set per shell."""
    atoms = np.asarray(mol.atoms, dtype=np.float64)
    shells = mol.shells
    ns = len(shells)
    maxp = max(len(s[2]) for s in shells)
    E = np.zeros((maxp, ns), order="F")
    Cf = np.zeros((maxp, ns), order="F")
    for i, s in enumerate(shells):
        E[:len(s[2]), i] = s[2]
        Cf[:len(s[3]), i] = s[3]
    L = np.array([s[1] for s in shells], dtype=np.int64)
    npr = np.array([len(s[2]) for s in shells], dtype=np.int64)
    ncart_n, nsph_n = basis_NormalizeCntrCoeffs(Cf, E, npr, L)
    return basis_Init_2(atoms.T, np.array([s[0] + 1 for s in shells]), np.arange(1, ns + 1), L, npr, Cf, E,
                        ncart_n, SpherAO=spher, NormFactorsSpher=nsph_n)
