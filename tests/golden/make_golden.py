"""Generate the golden fixtures of the parity tests from the reference's own
Python code (run in a container that has the reference source mounted).

* spherical_u.json -- Cartesian -> real solid harmonic coefficients for
  L = 0..5 from AutoSpherTransf.RSHU (src/integrals/Auto2e/AutoSpherTransf.py),
  rows m = -L..L (GabIndexSpher order, Auto2eGlobal.py:112-118), columns in the
  Auto2e Cartesian order (Auto2eGlobal.AngularFunctions, :35-44).
* index_tables.json -- the reference's Cartesian and Hermite (tuv) orderings.
* boys.json -- F_m(x) to 30 digits (mpmath quadrature) on a grid of x and m,
  the ground truth behind the Boys error targets of boys.f90:27-43,96-97.

Usage: python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
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

    import mpmath as mp
    mp.mp.dps = 32
    xs = [0.0, 1e-8, 0.01, 0.3, 1.0, 2.5, 7.0, 12.0, 19.9, 24.99, 25.0, 25.01, 33.0, 60.0]
    ms = [0, 1, 2, 4, 6, 8, 10, 12, 16, 20]
    vals = {}
    for m in ms:
        vals[str(m)] = [float(mp.quad(lambda t: t ** (2 * m) * mp.e ** (-x * t * t), [0, 1])) for x in xs]
    (HERE / "boys.json").write_text(json.dumps({"x": xs, "F": vals, "method": "mpmath.quad, 32 digits"}))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
