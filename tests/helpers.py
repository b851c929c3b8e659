"""Shared helpers of the parity tests: build the same molecule for the
library (TAOBasis) and the oracle (raw shells)."""
import numpy as np

from gammcor_integrals_b200 import basis as gbasis
from gammcor_integrals_b200 import molecules
from oracle import oracle as O


def both(mol, spher=True):
    return gbasis.from_molecule(mol, spher=spher), O.make_basis(mol.atoms, mol.shells, spher=spher)


def full_order_pairs(nshellpairs, shellpairs0, ob):
    """(p, q) AO indices (0-based) of each orbital pair in FULL storage order.
    shellpairs0: (nsp, 2) 0-based shells (A >= B)."""
    out = []
    for s in range(nshellpairs):
        A, B = shellpairs0[s]
        Na = 2 * int(ob.L[A]) + 1 if ob.spher else (int(ob.L[A]) + 1) * (int(ob.L[A]) + 2) // 2
        Nb = 2 * int(ob.L[B]) + 1 if ob.spher else (int(ob.L[B]) + 1) * (int(ob.L[B]) + 2) // 2
        for b in range(Nb):
            for a in range(b if A == B else 0, Na):
                out.append((ob.shell_loc[A] + a, ob.shell_loc[B] + b))
    return np.array(out)


def vectors_full_order(Rkpq, shellpairloc_1based, shellpairdim):
    """(NVecs, NOrbPairs) Cholesky vectors with columns in FULL order."""
    nv = Rkpq.shape[0]
    npq = int(np.sum(shellpairdim))
    R = np.zeros((nv, npq))
    for s in range(len(shellpairdim)):
        full, sub, X = (int(v) - 1 for v in shellpairloc_1based[:, s])
        d = int(shellpairdim[s])
        R[:, full:full + d] = Rkpq[:, sub:sub + d, X]
    return R
