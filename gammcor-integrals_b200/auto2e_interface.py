"""AO-ordering conversion between external programs and the Auto2e order.

Mirrors module Auto2eInterface (src/gammcor-interface/Auto2eInterface.f90):
the ORBITAL_ORDERING_* constants (:12-17), the per-L position tables of each
program (:27-213), auto2e_interface_AngFuncTransf (:217-275),
auto2e_interface_AOMap (:378-514) and the ORCA phase convention (:517-585).
Within a shell the Auto2e order is m = -L..L for L >= 2 and (x, y, z) for p.
The tables give, for each external position, the Auto2e position (1-based).
"""
from __future__ import annotations

import numpy as np

ORBITAL_ORDERING_AUTO2E = 0
ORBITAL_ORDERING_MOLPRO = 1
ORBITAL_ORDERING_ORCA = 2
ORBITAL_ORDERING_DALTON = 3
ORBITAL_ORDERING_OPEN_MOLCAS = 4
ORBITAL_ORDERING_PYSCF = 5


def _m(ms, L):
    """Auto2e positions (1-based) of the listed m values of an L shell."""
    return [m + L + 1 for m in ms]


_P_XYZ = [1, 2, 3]
_MINUS_L_TO_L = {L: _m(range(-L, L + 1), L) for L in range(2, 6)}

SPHER_MAPS = {
    ORBITAL_ORDERING_MOLPRO: {0: [1], 1: _P_XYZ,
                              2: _m([0, -2, 1, 2, -1], 2),
                              3: _m([1, -1, 0, 3, -2, -3, 2], 3),
                              4: _m([0, -2, 1, 4, -1, 2, -4, 3, -3], 4),
                              5: _m([1, -1, 2, 3, -4, -3, 4, -5, 0, 5, -2], 5)},
    ORBITAL_ORDERING_ORCA: {0: [1], 1: [3, 1, 2],
                            2: _m([0, 1, -1, 2, -2], 2),
                            3: _m([0, 1, -1, 2, -2, 3, -3], 3),
                            4: _m([0, 1, -1, 2, -2, 3, -3, 4, -4], 4),
                            5: _m([0, 1, -1, 2, -2, 3, -3, 4, -4, 5, -5], 5)},
    ORBITAL_ORDERING_DALTON: {0: [1], 1: _P_XYZ, **_MINUS_L_TO_L},
    ORBITAL_ORDERING_PYSCF: {0: [1], 1: _P_XYZ, **_MINUS_L_TO_L},
    ORBITAL_ORDERING_OPEN_MOLCAS: {0: [1], 1: _P_XYZ, **_MINUS_L_TO_L},
}

# Cartesian Molpro order, Auto2eInterface.f90:144-213
CART_MAPS_MOLPRO = {0: [1], 1: [1, 2, 3], 2: [1, 4, 6, 2, 3, 5], 3: [1, 7, 10, 2, 3, 4, 8, 6, 9, 5],
                    4: [1, 11, 15, 2, 3, 7, 12, 10, 14, 4, 6, 13, 5, 8, 9], 5: list(range(1, 22))}


def auto2e_interface_AOMap(AOBasis, ExternalOrdering):
    """Map_extao2ao and Map_ao2extao (1-based), auto2e_interface_AOMap (:378-514)."""
    nao = AOBasis.NAO
    m_ext = np.full(nao, -1, dtype=np.int64)
    sh_params = AOBasis.ShellParamsIdx - 1
    Ls = AOBasis.ShellMomentum[sh_params]
    if AOBasis.SpherAO:
        if ExternalOrdering not in SPHER_MAPS:
            raise ValueError("Invalid external orbital ordering")
        tab = SPHER_MAPS[ExternalOrdering]
        loc = AOBasis.ShellLocSpher
        if ExternalOrdering == ORBITAL_ORDERING_OPEN_MOLCAS:
            # within an atom: all functions of one L, ordered by M, then by shell
            for a in range(1, AOBasis.NAtoms + 1):
                shells = np.nonzero(AOBasis.ShellCenters == a)[0]
                if shells.size == 0:
                    continue
                s0, s1 = shells[0], shells[-1]
                i = loc[s0]
                for L in range(int(Ls[s0:s1 + 1].max()) + 1):
                    for M in range(2 * L + 1):
                        for s in range(s0, s1 + 1):
                            if Ls[s] == L:
                                m_ext[i - 1] = loc[s] + tab[L][M] - 1
                                i += 1
        else:
            for s in range(AOBasis.NShells):
                L = int(Ls[s])
                p0 = loc[s]
                for k, pos in enumerate(tab[L]):
                    m_ext[p0 - 1 + k] = p0 + pos - 1
    else:
        if ExternalOrdering != ORBITAL_ORDERING_MOLPRO:
            raise ValueError("Invalid external orbital ordering")
        loc = AOBasis.ShellLocCart
        for s in range(AOBasis.NShells):
            L = int(Ls[s])
            p0 = loc[s]
            for k, pos in enumerate(CART_MAPS_MOLPRO[L]):
                m_ext[p0 - 1 + k] = p0 + pos - 1
    m_ao = np.zeros(nao, dtype=np.int64)
    m_ao[m_ext - 1] = np.arange(1, nao + 1)
    return m_ext, m_ao


def auto2e_interface_AngFuncTransf(X_in, FromExternalAO: bool, TwoIndexTransf: bool, AOBasis, ExternalOrdering):
    """auto2e_interface_AngFuncTransf (:217-275); returns X_out."""
    X_in = np.asarray(X_in, dtype=np.float64)
    if ExternalOrdering == ORBITAL_ORDERING_AUTO2E:
        return np.array(X_in, order="F", copy=True)
    m_ext, m_ao = auto2e_interface_AOMap(AOBasis, ExternalOrdering)
    Map = (m_ext if FromExternalAO else m_ao) - 1
    X_out = np.zeros_like(X_in, order="F")
    if TwoIndexTransf:
        W = np.zeros_like(X_in)
        W[Map, :] = X_in
        X_out[:, Map] = W
    else:
        X_out[Map, :] = X_in
    return X_out


def _orca_positions(AOBasis):
    pos = []
    for s in range(AOBasis.NShells):
        L = int(AOBasis.ShellMomentum[AOBasis.ShellParamsIdx[s] - 1])
        base = AOBasis.ShellLocSpher[s] - 1
        if L >= 3:
            pos += [base + L + 3, base + L - 3]
        if L >= 4:
            pos += [base + L + 4, base + L - 4]
    return np.array(pos, dtype=np.int64)


def auto2e_interface_ApplyOrcaPhases_Matrix(X, AOBasis, TwoIndexTransf: bool):
    """ORCA sign convention for m = +-3, +-4 of f, g, h shells (:517-585).

    The reference flips rows of the first NAO columns (and, for two-index
    matrices, the matching columns)."""
    X = np.array(X, order="F", copy=True)
    p = _orca_positions(AOBasis)
    nao = X.shape[0]
    ncol = min(nao, X.shape[1])
    X[p, :ncol] *= -1.0
    if TwoIndexTransf:
        X[:, p] *= -1.0
    return X
