"""Generate the golden fixtures of the parity tests from the reference's own
Python code (run in a container that has the reference source mounted).

* spherical_u.json -- Cartesian -> real solid harmonic coefficients for
  L = 0..5 from AutoSpherTransf.RSHU (src/integrals/Auto2e/AutoSpherTransf.py),
  rows m = -L..L (GabIndexSpher order, Auto2eGlobal.py:112-118), columns in the
  Auto2e Cartesian order (Auto2eGlobal.AngularFunctions, :35-44).
* index_tables.json -- the reference's Cartesian and Hermite (tuv) orderings.
* boys.json -- F_m(x) to 30 digits (mpmath quadrature) on a grid of x and m,
  the ground truth behind the Boys error targets of boys.f90:27-43,96-97.
* hermite_recurrences.json -- the Hermite Coulomb integrals R_tuv and the
  Hermite expansion coefficients E^{l,0}_t evaluated by the straight-line
  statements the reference's generator emits (Auto2e.RtuvSubroutine /
  RtuvKSubroutine, Auto2e.py:80-119,1027-1066, and Auto2e.EtSubroutine,
  :997-1025), interpreted here at seeded inputs.

Usage: python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import re
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main(ref_root: str) -> None:
    auto2e = Path(ref_root) / "src" / "integrals" / "Auto2e"
    sys.path.insert(0, str(auto2e))
    # importing the generator writes its Fortran output under ./src; keep that
    # out of this tree by importing from a scratch directory
    here = os.getcwd()
    os.chdir(tempfile.mkdtemp(prefix="auto2e_gen_"))
    import Auto2eGlobal as G        # noqa: E402  (reference module)
    import AutoSpherTransf as AST   # noqa: E402  (reference module)
    import Auto2e as A2E            # noqa: E402  (reference module: tuvindices)
    os.chdir(here)

    U = {}
    for L in range(0, 6):
        carts = G.AngularFunctions[L]
        rows = []
        for m in range(-L, L + 1):
            u = AST.RSHU(L, m, L)
            rows.append([float(u[x][y][z]) for (x, y, z) in carts])
        U[str(L)] = rows
    (HERE / "spherical_u.json").write_text(json.dumps({"source": "AutoSpherTransf.RSHU(l, m, l)", "U": U}))

    tables = {"cartesian": {str(L): G.AngularFunctions[L] for L in range(0, 11)},
              "tuv": {str(n): sorted(((int(i), list(k)) for k, i in A2E.tuvindices(n).items()))
                      for n in range(0, 13)}}
    (HERE / "index_tables.json").write_text(json.dumps(tables))

    (HERE / "hermite_recurrences.json").write_text(json.dumps(recurrences(A2E, G), indent=None))

    import mpmath as mp
    mp.mp.dps = 32
    xs = [0.0, 1e-8, 0.01, 0.3, 1.0, 2.5, 7.0, 12.0, 19.9, 24.99, 25.0, 25.01, 33.0, 60.0]
    ms = [0, 1, 2, 4, 6, 8, 10, 12, 16, 20]
    vals = {}
    for m in ms:
        vals[str(m)] = [float(mp.quad(lambda t: t ** (2 * m) * mp.e ** (-x * t * t), [0, 1])) for x in xs]
    (HERE / "boys.json").write_text(json.dumps({"x": xs, "F": vals, "method": "mpmath.quad, 32 digits"}))


def _fortran_rhs(expr: str) -> str:
    """A right-hand side of the generated Fortran as a Python expression over the
    dicts RA, RB, E, Fm (1-based keys as in the Fortran arrays)."""
    expr = expr.replace("_F64", "")
    return re.sub(r"\b(RA|RB|E|Fm)\(([^()]*)\)", r"\1[\2]", expr)


def _run_rtuvk(code: str, RA: dict, RB: dict, n: int, Fm: dict, X, Y, Z, p) -> None:
    for line in code.splitlines():
        m = re.match(r"^RA\((\d+)\) = (.*)$", line.strip())
        if m:
            RA[int(m.group(1))] = eval(_fortran_rhs(m.group(2)), {}, {"RB": RB, "Fm": Fm, "X": X, "Y": Y, "Z": Z,
                                                                    "p": p, "n": n})


def _run_rtuv(n: int, A2E, Fm: dict, X, Y, Z, p) -> dict:
    """auto2e_Rtuv_n as emitted by RtuvSubroutine(n): a seed statement and calls of
    auto2e_RtuvK_k, each interpreted statement by statement."""
    arrays = {"RA": {}, "RB": {}}
    for line in A2E.RtuvSubroutine(n).splitlines():
        line = line.strip()
        m = re.match(r"^(RA|RB)\(1\) = (.*)$", line)
        if m:
            arrays[m.group(1)][1] = eval(_fortran_rhs(m.group(2)), {}, {"Fm": Fm, "p": p})
            continue
        m = re.match(r"^call auto2e_RtuvK_(\d+)\((RA|RB), (RA|RB), (\d+), Fm, X, Y, Z, p\)$", line)
        if m:
            k, out, inp, nn = int(m.group(1)), m.group(2), m.group(3), int(m.group(4))
            res = {}
            _run_rtuvk(A2E.RtuvKSubroutine(k), res, arrays[inp], nn, Fm, X, Y, Z, p)
            arrays[out] = res
    return arrays["RA"]


def _run_et(L: int, A2E, p, X, E000) -> dict:
    E = {}
    for line in A2E.EtSubroutine(L).splitlines():
        m = re.match(r"^E\((\d+)\) = (.*)$", line.strip())
        if m:
            E[int(m.group(1))] = eval(_fortran_rhs(m.group(2)), {}, {"E": E, "p": p, "X": X, "E000": E000})
    return E


def recurrences(A2E, G) -> dict:
    rng = np.random.default_rng(2024)
    rcases = []
    for n in range(0, 13):
        for _ in range(2):
            alpha = float(np.exp(rng.uniform(np.log(0.05), np.log(50.0))))
            X, Y, Z = (float(v) for v in rng.uniform(-2.0, 2.0, 3))
            F = [float(v) for v in np.sort(rng.uniform(0.01, 1.0, n + 1))[::-1]]
            R = _run_rtuv(n, A2E, {m + 1: F[m] for m in range(n + 1)}, X, Y, Z, alpha)
            tuv = A2E.tuvindices(n)
            rcases.append({"n": n, "alpha": alpha, "X": X, "Y": Y, "Z": Z, "F": F,
                           "R": [[t, u, v, float(R[i])] for (t, u, v), i in sorted(tuv.items(), key=lambda x: x[1])]})
    ecases = []
    for L in range(0, 2 * G.MaxL + 1):
        p = float(np.exp(rng.uniform(np.log(0.05), np.log(5e3))))
        X = float(rng.uniform(-2.0, 2.0))
        E = _run_et(L, A2E, p, X, 1.0)
        ecases.append({"L": L, "p": p, "X": X,
                       "E": [[l, t, float(E[G.EtIdx[(l, t)]])] for l in range(L + 1) for t in range(l + 1)]})
    return {"source": "Auto2e.RtuvSubroutine/RtuvKSubroutine and Auto2e.EtSubroutine statements, interpreted",
            "rtuv": rcases, "et": ecases}


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/reference")
    main(sys.argv[1])
