"""Import helper for the package directory ``gammcor-integrals_b200``.

The directory name is not a valid Python identifier, so the package is
registered as ``gammcor_integrals_b200`` by path.
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

PKG_NAME = "gammcor_integrals_b200"
PKG_DIR = Path(__file__).resolve().parent / "gammcor-integrals_b200"


def load():
    if PKG_NAME in sys.modules:
        return sys.modules[PKG_NAME]
    spec = importlib.util.spec_from_file_location(PKG_NAME, PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[PKG_NAME] = mod
    spec.loader.exec_module(mod)
    return mod
