"""Host-side mirror of the reference's Gammcor Cholesky interface.

Mirrors module Cholesky_Gammcor (src/gammcor-interface/Cholesky_Gammcor.f90):
the CHOL_ACCURACY_* constants (:14-17), TCholeskyVecsOTF (:19-22),
chol_gammcor_Rkpq (:335-377) and chol_gammcor_Rkab (:26-92), with TChol2Vecs
of TwoStepCholesky_definitions (:56-74).  All compute runs in libgci.so on the
GPU; errors the reference turns into ``error stop`` raise GciError here.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from .auto2e_interface import ORBITAL_ORDERING_AUTO2E, auto2e_interface_AngFuncTransf, \
    auto2e_interface_ApplyOrcaPhases_Matrix, ORBITAL_ORDERING_ORCA
from .basis import TAOBasis

CHOL_ACCURACY_DEFAULT = 1
CHOL_ACCURACY_TIGHT = 2
CHOL_ACCURACY_LUDICROUS = 3
CHOL_ACCURACY_DEBUG = 4


@dataclass
class TChol2Vecs:
    """TChol2Vecs (TwoStepCholesky_definitions.f90:56-74), 1-based indices."""
    Inv_L: np.ndarray
    NVecs: int
    MaxSubsetDim: int
    NSubsets: np.ndarray
    NOrbPairs: int
    NShellPairs: int
    ShellPairs: np.ndarray
    ShellPairLoc: np.ndarray
    ShellPairDim: np.ndarray
    SubsetDim: np.ndarray
    SubsetBounds: np.ndarray
    Pivots: np.ndarray
    PivotShellPairs: np.ndarray
    PivotShellPairLoc: np.ndarray
    PivotShellPairDim: np.ndarray
    PivotOrbPairs: np.ndarray
    NPivotShellPairs: int


@dataclass
class TCholeskyVecsOTF:
    """TCholeskyVecsOTF (Cholesky_Gammcor.f90:19-22).  ``Rkpq`` is the host
    copy (NVecs, MaxSubsetDim, NSubsets) when it was materialised; the device
    state stays behind ``handle`` for chol_gammcor_Rkab."""
    Rkpq: np.ndarray | None
    Chol2Data: TChol2Vecs
    handle: "_Handle" = field(repr=False, default=None)
    pivot_order: np.ndarray | None = None
    pivot_dmax: np.ndarray | None = None

    def timings(self) -> dict:
        return self.handle.timings()


class _Handle:
    def __init__(self, ptr: C.c_void_p):
        self.ptr = ptr

    def __del__(self):
        if getattr(self, "ptr", None):
            try:
                _capi.lib().gci_free(self.ptr)
            except Exception:
                pass
            self.ptr = None

    def timings(self) -> dict:
        out = np.zeros(13)
        _capi.check(_capi.lib().gci_timings(self.ptr, _capi.ptr(out), 13))
        keys = ["vdiag", "step1_eri", "subtract_r", "pivots", "compress", "vjj_eri", "potrf_trtri", "fulldim_eri",
                "invl_gemm", "mo_gemm", "n_macro", "rkpq_wall", "rkab_wall"]
        return dict(zip(keys, out.tolist()))


def accuracy_tau(Accuracy: int) -> float:
    return {CHOL_ACCURACY_DEFAULT: 1e-5, CHOL_ACCURACY_TIGHT: 1e-6, CHOL_ACCURACY_LUDICROUS: 1e-7,
            CHOL_ACCURACY_DEBUG: 1e-10}[Accuracy]


def chol_gammcor_Rkpq(AOBasis: TAOBasis, Accuracy: int, Omega: float | None = None, *, materialize: bool = True,
                      copy_to_host: bool = True, decode_storage: bool = False,
                      mixed_step1: bool = False) -> TCholeskyVecsOTF:
    """Cholesky vectors in the AO basis computed on the fly (Cholesky_Gammcor.f90:335-377).
    mixed_step1: M - L L^T of the pivot search as a split-precision int8 tensor-core GEMM."""
    L = _capi.lib()
    b = AOBasis.c_struct()
    flags = (_capi.GCI_FLAG_MATERIALIZE_RKPQ if materialize else 0) | \
            (_capi.GCI_FLAG_PIVOT_DECODE_STORAGE if decode_storage else 0) | \
            (_capi.GCI_FLAG_MIXED_STEP1 if mixed_step1 else 0)
    h = C.c_void_p()
    _capi.check(L.gci_rkpq(C.byref(b), int(Accuracy), float(Omega) if Omega else 0.0, flags, C.byref(h)))
    return _vecs_from_handle(_Handle(h), materialize and copy_to_host)


def chol_gammcor_Rkpq_batch(AOBases, Accuracy: int, Omega: float | None = None, *, materialize: bool = True,
                            copy_to_host: bool = True, nstreams: int = 16) -> list:
    """chol_gammcor_Rkpq for many independent molecules in one call (gci_rkpq_batch): the
    molecules run concurrently, one CUDA stream per worker.  Returns one TCholeskyVecsOTF per basis."""
    L = _capi.lib()
    n = len(AOBases)
    views = [tb.c_struct() for tb in AOBases]   # each keeps its arrays alive; the array below copies pointers
    structs = (_capi.gci_basis * n)(*views)
    flags = _capi.GCI_FLAG_MATERIALIZE_RKPQ if materialize else 0
    hs = (C.c_void_p * n)()
    _capi.check(L.gci_rkpq_batch(n, structs, int(Accuracy), float(Omega) if Omega else 0.0, flags, int(nstreams),
                                 hs))
    out = [_vecs_from_handle(_Handle(C.c_void_p(hs[i])), materialize and copy_to_host) for i in range(n)]
    del views
    return out


def _vecs_from_handle(handle: "_Handle", copy_rkpq: bool) -> TCholeskyVecsOTF:
    L = _capi.lib()
    h = handle.ptr
    dims = [C.c_int64() for _ in range(6)]
    _capi.check(L.gci_query(h, *[C.byref(d) for d in dims]))
    nvecs, msd, nsub, npq, nsp, npsp = (d.value for d in dims)
    i64 = lambda n: np.zeros(max(n, 0), dtype=np.int64)
    sp, spl, spd = i64(2 * nsp), i64(3 * nsp), i64(nsp)
    sd, sb, piv = i64(nsub), i64(2 * nsub), i64(npq)
    psp, pspl, pspd, porb = i64(npsp), i64(npsp), i64(npsp), i64(nvecs)
    invl = np.zeros((nvecs, nvecs), order="F")
    P = lambda a: _capi.ptr(a, _capi._pl)
    _capi.check(L.gci_copy_chol2data(h, P(sp), P(spl), P(spd), P(sd), P(sb), P(piv), P(psp), P(pspl), P(pspd),
                                     P(porb), _capi.ptr(invl)))
    order, dm = i64(nvecs), np.zeros(nvecs)
    _capi.check(L.gci_pivot_order(h, P(order), _capi.ptr(dm)))
    chol2 = TChol2Vecs(Inv_L=invl, NVecs=nvecs, MaxSubsetDim=msd, NSubsets=np.array([nsub, 1]), NOrbPairs=npq,
                       NShellPairs=nsp, ShellPairs=sp.reshape(nsp, 2).T, ShellPairLoc=spl.reshape(nsp, 3).T,
                       ShellPairDim=spd, SubsetDim=sd, SubsetBounds=sb.reshape(nsub, 2).T, Pivots=piv,
                       PivotShellPairs=psp, PivotShellPairLoc=pspl, PivotShellPairDim=pspd, PivotOrbPairs=porb,
                       NPivotShellPairs=npsp)
    rkpq = None
    if copy_rkpq:
        rkpq = np.zeros((nvecs, msd, nsub), order="F")
        _capi.check(L.gci_copy_rkpq(h, _capi.ptr(rkpq)))
    return TCholeskyVecsOTF(Rkpq=rkpq, Chol2Data=chol2, handle=handle, pivot_order=order, pivot_dmax=dm)


def chol_gammcor_Rkab(CA: np.ndarray, a0: int, a1: int, CB: np.ndarray, b0: int, b1: int, MaxBufferDimMB: int,
                      CholeskyVecsOTF: TCholeskyVecsOTF, AOBasis: TAOBasis,
                      ExternalOrdering: int = ORBITAL_ORDERING_AUTO2E, *, precision: str = "fp64",
                      Rkab: np.ndarray | None = None) -> np.ndarray:
    """Transformation of the Cholesky vectors to the MO basis (Cholesky_Gammcor.f90:26-92).

    a0..a1 and b0..b1 are 1-based inclusive column ranges of CA and CB.
    Returns Rkab(NVecs, NA*NB), k fastest, then a, then b."""
    NA, NB = a1 - a0 + 1, b1 - b0 + 1
    nvecs = CholeskyVecsOTF.Chol2Data.NVecs
    nao = AOBasis.NAO
    if CA.shape[0] != nao or CB.shape[0] != nao:
        raise _capi.GciError(-1, "Invalid number of atomic orbitals in CA/CB")
    if Rkab is not None and (Rkab.shape[0] != nvecs or Rkab.shape[1] != NA * NB):
        raise _capi.GciError(-1, "Invalid dimension of Rkab")
    CA_ao = auto2e_interface_AngFuncTransf(np.asfortranarray(CA, dtype=np.float64), True, False, AOBasis,
                                           ExternalOrdering)
    CB_ao = auto2e_interface_AngFuncTransf(np.asfortranarray(CB, dtype=np.float64), True, False, AOBasis,
                                           ExternalOrdering)
    if ExternalOrdering == ORBITAL_ORDERING_ORCA:
        CA_ao = auto2e_interface_ApplyOrcaPhases_Matrix(CA_ao, AOBasis, False)
        CB_ao = auto2e_interface_ApplyOrcaPhases_Matrix(CB_ao, AOBasis, False)
    prec = {"fp64": _capi.GCI_PREC_FP64, "mixed": _capi.GCI_PREC_MIXED}[precision]
    out = Rkab if Rkab is not None else np.zeros((nvecs, NA * NB), order="F")
    assert out.flags.f_contiguous and out.dtype == np.float64
    CA_ao = np.asfortranarray(CA_ao)
    CB_ao = np.asfortranarray(CB_ao)
    _capi.check(_capi.lib().gci_rkab(CholeskyVecsOTF.handle.ptr, _capi.ptr(CA_ao), CA_ao.shape[0], a0, a1,
                                     _capi.ptr(CB_ao), CB_ao.shape[0], b0, b1, int(MaxBufferDimMB), prec,
                                     _capi.ptr(out)))
    return out
