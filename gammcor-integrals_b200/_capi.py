"""ctypes binding of libgci.so (include/gci.h).

The library is required: importing the compute entry points without it, or
calling them without a CUDA device, raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_lib" / "libgci.so"

GCI_OK = 0
GCI_ACCURACY_DEFAULT, GCI_ACCURACY_TIGHT, GCI_ACCURACY_LUDICROUS, GCI_ACCURACY_DEBUG = 1, 2, 3, 4
GCI_FLAG_MATERIALIZE_RKPQ = 1
GCI_FLAG_PIVOT_DECODE_STORAGE = 2
GCI_FLAG_MIXED_STEP1 = 4
GCI_PREC_FP64, GCI_PREC_MIXED = 0, 1
GCI_ERR_BUFFER = -6
GCI_NOALLOC_SCRATCH_BYTES = 16 << 20

# every entry point declared in include/gci.h
EXPORTS = ("gci_init", "gci_rkpq", "gci_query", "gci_copy_rkpq", "gci_copy_chol2data", "gci_pivot_order",
           "gci_rkab", "gci_timings", "gci_free", "gci_last_error", "gci_boys", "gci_spher_coeffs",
           "gci_normalize_basis", "gci_eri_pairs", "gci_rkab_device", "gci_stats", "gci_get_stream",
           "gci_kernel_launches", "gci_eri_pairs_noalloc", "gci_eri_variant", "gci_eri_hm", "gci_eri_hm_stats", "gci_rkpq_columns", "gci_dgemm_split",
           "gci_dgemm", "gci_cholesky_inverse", "gci_trsm_rlt", "gci_autotune_eri",
           "gci_coulomb_grad", "gci_coulomb_grad_device", "gci_coulomb_grad_work", "gci_rkpq_batch")

_pd = C.POINTER(C.c_double)
_pl = C.POINTER(C.c_int64)
_i64 = C.c_int64


class GciError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libgci error {code}: {msg}")
        self.code = code


class gci_basis(C.Structure):
    _fields_ = [("natoms", _i64), ("nshells", _i64), ("nshellparams", _i64), ("ldprim", _i64), ("ldnorm", _i64),
                ("atom_coords", _pd), ("shell_centers", _pl), ("shell_params_idx", _pl),
                ("shell_momentum", _pl), ("nprimitives", _pl), ("cntr_coeffs", _pd), ("exponents", _pd),
                ("norm_factors", _pd), ("spher_ao", C.c_int32)]


_lib = None


def lib():
    """Load libgci.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with build_lib.py (nvcc, sm_100a)")
        L = C.CDLL(str(LIB_PATH))
        L.gci_init.argtypes = []
        L.gci_rkpq.argtypes = [C.POINTER(gci_basis), C.c_int, C.c_double, C.c_int, C.POINTER(C.c_void_p)]
        L.gci_rkpq_batch.argtypes = [_i64, C.POINTER(gci_basis), C.c_int, C.c_double, C.c_int, C.c_int,
                                     C.POINTER(C.c_void_p)]
        L.gci_query.argtypes = [C.c_void_p] + [_pl] * 6
        L.gci_copy_rkpq.argtypes = [C.c_void_p, _pd]
        L.gci_copy_chol2data.argtypes = [C.c_void_p] + [_pl] * 10 + [_pd]
        L.gci_pivot_order.argtypes = [C.c_void_p, _pl, _pd]
        L.gci_rkab.argtypes = [C.c_void_p, _pd, _i64, _i64, _i64, _pd, _i64, _i64, _i64, _i64, C.c_int, _pd]
        L.gci_timings.argtypes = [C.c_void_p, _pd, C.c_int]
        L.gci_free.argtypes = [C.c_void_p]
        L.gci_free.restype = None
        L.gci_last_error.restype = C.c_char_p
        L.gci_boys.argtypes = [C.c_int, _i64, _pd, _pd]
        L.gci_spher_coeffs.argtypes = [C.c_int, _pd]
        L.gci_normalize_basis.argtypes = [_i64, _i64, _pl, _pl, _pd, _pd, _pd, _i64, _pd, _i64]
        L.gci_eri_pairs.argtypes = [C.POINTER(gci_basis), C.c_double, _pd, _i64]
        L.gci_rkab_device.argtypes = [C.c_void_p, C.c_void_p, _i64, _i64, _i64, C.c_void_p, _i64, _i64, _i64, _i64,
                                      C.c_int, C.c_void_p]
        L.gci_stats.argtypes = [C.c_void_p, _pd, C.c_int]
        L.gci_get_stream.argtypes = [C.POINTER(C.c_void_p)]
        L.gci_kernel_launches.argtypes = [_pl]
        L.gci_eri_variant.argtypes = [C.c_int, C.c_int, C.c_int]
        L.gci_eri_hm.argtypes = [C.c_int]
        L.gci_eri_hm_stats.argtypes = [C.c_void_p, _pd, C.c_int]
        L.gci_rkpq_columns.argtypes = [C.c_void_p, _i64, _pl, _pd]
        L.gci_dgemm_split.argtypes = [_i64, _i64, _i64, C.c_double, C.c_void_p, _i64, C.c_void_p, _i64, C.c_double,
                                      C.c_void_p, _i64]
        L.gci_dgemm.argtypes = L.gci_dgemm_split.argtypes
        L.gci_cholesky_inverse.argtypes = [_i64, C.c_void_p, _i64, C.c_void_p]
        L.gci_trsm_rlt.argtypes = [_i64, _i64, C.c_void_p, _i64, C.c_void_p, _i64]
        L.gci_autotune_eri.argtypes = [C.POINTER(gci_basis), C.c_int, _pd]
        L.gci_coulomb_grad.argtypes = [C.POINTER(gci_basis), C.c_double, _pd, _i64, _pd, _pd, _pd, _i64]
        L.gci_coulomb_grad_device.argtypes = [C.POINTER(gci_basis), C.c_double, C.c_void_p, _i64, _pd, _pd,
                                              C.c_void_p, _i64]
        L.gci_coulomb_grad_work.argtypes = [_pd, C.c_int]
        L.gci_eri_pairs_noalloc.argtypes = [C.POINTER(gci_basis), C.c_double, C.c_void_p, _i64, C.c_void_p]
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != GCI_OK:
        raise GciError(rc, lib().gci_last_error().decode())


def ptr(a: np.ndarray, t=_pd):
    return a.ctypes.data_as(t) if a is not None else None
