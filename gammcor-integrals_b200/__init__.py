"""B200-native integral-direct Cholesky decomposition of the Coulomb ERI
matrix and AO->MO transformation of the Cholesky vectors.

A drop-in for the Gammcor interface of modrzejewski/gammcor-integrals
(src/gammcor-interface/Cholesky_Gammcor.f90): the compute runs in libgci.so
(hand-written sm_100a kernels behind a C ABI, include/gci.h); this package
is the host-side mirror of the reference's Fortran interface.
"""
from __future__ import annotations

__version__ = "0.1.0"
