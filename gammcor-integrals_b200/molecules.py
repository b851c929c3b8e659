"""Seeded synthetic molecules for the benchmark configurations.

There is no public data set for this path; the workloads are random
molecules with the shapes and value distributions of the five
configurations of the integral-direct Cholesky benchmark:

* ``c1`` 10 atoms, 8 bohr cube, shells s,s,s,p,p,d, 3 primitives, exponents
  log-uniform in [0.1, 1e3] (140 spherical AOs), tau = 1e-6, MO 20 x 60.
* ``c2`` 40 atoms, 16 bohr cube, shells s x4, p x3, d x2, f, 3-6 primitives,
  exponents log-uniform in [0.05, 5e3] (1200 AOs), tau = 1e-6, MO 60 x 900.
* ``c3`` 64 molecules of 3-30 atoms (8 bohr cube), the c1 recipe, tau = 1e-5.
* ``c4`` 20 atoms, 12 bohr cube, the c1 recipe (280 AOs); density X X^T with
  X ~ N(0, 0.1^2), 280 x 30.
* ``c5`` 120 atoms, 24 bohr cube, the c2 recipe (3600 AOs), MO 150 x 2700.
* ``c2s`` 12 atoms with the c2 recipe at the c2 atom density (360 AOs),
  MO 18 x 270: the same kernels as c2 on a case small enough to profile.

Atoms are placed uniformly in the cube and rejected when closer than
1.7 bohr to an accepted atom; contraction coefficients are N(0, 1) before
normalisation.  A molecule is a plain description -- ``atoms`` (natoms, 3)
in bohr and ``shells`` = [(atom, L, exponents, raw coefficients)] -- that
both the library and the CPU oracle consume.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

RECIPE_C1 = (0, 0, 0, 1, 1, 2)
RECIPE_C2 = (0, 0, 0, 0, 1, 1, 1, 2, 2, 3)


@dataclass
class Molecule:
    atoms: np.ndarray            # (natoms, 3) bohr
    shells: list                 # [(atom, L, exps, coefs)]
    tau: float = 1e-6
    name: str = ""

    @property
    def nao(self) -> int:
        return sum(2 * s[1] + 1 for s in self.shells)

    @property
    def nshells(self) -> int:
        return len(self.shells)


def place_atoms(rng: np.random.Generator, natoms: int, cube: float, dmin: float = 1.7,
                max_tries: int = 1_000_000) -> np.ndarray:
    pts = []
    tries = 0
    while len(pts) < natoms:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place atoms with the requested minimum distance")
        p = rng.uniform(0.0, cube, 3)
        if all(np.linalg.norm(p - q) >= dmin for q in pts):
            pts.append(p)
    return np.array(pts)


def random_molecule(seed: int, natoms: int, cube: float, recipe=RECIPE_C1, nprim=(3, 3),
                    exp_range=(0.1, 1.0e3), tau: float = 1e-6, name: str = "") -> Molecule:
    rng = np.random.default_rng(seed)
    atoms = place_atoms(rng, natoms, cube)
    lo, hi = np.log(exp_range[0]), np.log(exp_range[1])
    shells = []
    for a in range(natoms):
        for L in recipe:
            n = int(rng.integers(nprim[0], nprim[1] + 1))
            exps = np.sort(np.exp(rng.uniform(lo, hi, n)))[::-1].copy()
            coefs = rng.standard_normal(n)
            shells.append((a, int(L), exps, coefs))
    return Molecule(atoms=atoms, shells=shells, tau=tau, name=name)


def config(name: str, index: int = 0) -> Molecule:
    """The benchmark molecules; ``index`` selects one of the 64 c3 molecules."""
    if name == "c1":
        return random_molecule(1, 10, 8.0, RECIPE_C1, (3, 3), (0.1, 1e3), 1e-6, "c1")
    if name == "c2":
        return random_molecule(2, 40, 16.0, RECIPE_C2, (3, 6), (0.05, 5e3), 1e-6, "c2")
    if name == "c2s":
        # the c2 recipe at the c2 atom density with 12 atoms (360 AOs): profiling-size case
        return random_molecule(2, 12, 16.0 * (12 / 40) ** (1 / 3), RECIPE_C2, (3, 6), (0.05, 5e3), 1e-6, "c2s")
    if name == "c3":
        counts = np.random.default_rng(3).integers(3, 31, 64)
        return random_molecule(3000 + index, int(counts[index]), 8.0, RECIPE_C1, (3, 3), (0.1, 1e3), 1e-5,
                               f"c3[{index}]")
    if name == "c4":
        return random_molecule(4, 20, 12.0, RECIPE_C1, (3, 3), (0.1, 1e3), 1e-6, "c4")
    if name == "c5":
        return random_molecule(5, 120, 24.0, RECIPE_C2, (3, 6), (0.05, 5e3), 1e-6, "c5")
    raise ValueError(f"unknown configuration {name!r}")


def mo_coefficients(nao: int, seed: int) -> np.ndarray:
    """Seeded orthonormal NAO x NAO matrix: Q of the QR of an N(0,1) matrix."""
    q, r = np.linalg.qr(np.random.default_rng(seed).standard_normal((nao, nao)))
    return np.asfortranarray(q * np.sign(np.diag(r)))


MO_SPLIT = {"c1": (20, 60, 101), "c2": (60, 900, 102), "c2s": (18, 270, 102), "c5": (150, 2700, 105)}


def small_molecule(seed: int, natoms: int = 3, recipe=RECIPE_C1, cube: float = 5.0, nprim=(3, 3),
                   exp_range=(0.1, 1.0e3), tau: float = 1e-6) -> Molecule:
    """A small molecule of the same kind, for parity tests."""
    return random_molecule(seed, natoms, cube, recipe, nprim, exp_range, tau, f"small{seed}")
