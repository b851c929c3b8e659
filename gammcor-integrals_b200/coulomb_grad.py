"""Coulomb energy of a density and its nuclear gradient on the GPU.

J = 1/2 sum_{pq,rs} D_pq (pq|rs) D_rs, dJ/dAtomCoords and the Coulomb matrix
J_pq = dJ/dD_pq come from libgci.so's adjoint kernels (gci_coulomb_grad*,
include/gci.h): derivative integrals by Hermite index shifts of the
McMurchie-Davidson scheme the reference's ERI engine uses
(src/integrals/Auto2e), contracted with the density in Hermite space.  The
reference has no derivative integrals; this is new.

``CoulombEnergy`` wraps the kernels as a ``torch.autograd.Function`` of the
atom coordinates and the density.  There is no CPU fallback: without the
library or a CUDA device the calls raise.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import replace

import numpy as np

from . import _capi


def coulomb_energy_grad(tb, D: np.ndarray, omega: float = 0.0, want_jmat: bool = False):
    """(J, grad (NAtoms, 3), Jmat or None) of the density D (NAO x NAO, AO order of ``tb``)
    through the host entry point gci_coulomb_grad."""
    L = _capi.lib()
    nao = tb.NAO
    D = np.asfortranarray(D, dtype=np.float64)
    if D.shape != (nao, nao):
        raise ValueError(f"D must be {nao} x {nao}")
    e = C.c_double(0.0)
    g = np.zeros((tb.NAtoms, 3))            # row-major (NAtoms, 3) == column-major (3, NAtoms)
    jm = np.zeros((nao, nao), order="F") if want_jmat else None
    s = tb.c_struct()
    _capi.check(L.gci_coulomb_grad(C.byref(s), omega, _capi.ptr(D), nao, C.byref(e), _capi.ptr(g),
                                   _capi.ptr(jm), nao))
    return e.value, g, jm


def with_coords(tb, coords: np.ndarray):
    """A copy of the basis with the atoms moved to ``coords`` (NAtoms, 3)."""
    return replace(tb, AtomCoords=np.asfortranarray(np.asarray(coords, dtype=np.float64).T))


def _device_call(tb, D, omega, want_jmat):
    import torch
    L = _capi.lib()
    nao = tb.NAO
    # D is symmetrised by the kernels, so its row-major storage read as
    # column-major (D^T) gives the same J, gradient and Coulomb matrix
    Dc = D.detach().to(dtype=torch.float64).contiguous()
    e = C.c_double(0.0)
    g = np.zeros((tb.NAtoms, 3))
    jm = torch.empty((nao, nao), dtype=torch.float64, device=Dc.device) if want_jmat else None
    s = tb.c_struct()
    cur = torch.cuda.current_stream(Dc.device)
    sptr = C.c_void_p()
    _capi.check(L.gci_get_stream(C.byref(sptr)))
    lib_stream = torch.cuda.ExternalStream(sptr.value, device=Dc.device)
    lib_stream.wait_stream(cur)
    _capi.check(L.gci_coulomb_grad_device(C.byref(s), omega, C.c_void_p(Dc.data_ptr()), nao, C.byref(e),
                                          _capi.ptr(g), C.c_void_p(jm.data_ptr()) if jm is not None else None, nao))
    cur.wait_stream(lib_stream)
    return e.value, g, jm


class CoulombEnergy:
    """torch.autograd.Function J(coords, D) = 1/2 sum D_pq (pq|rs) D_rs.

    ``coords`` (NAtoms, 3) in bohr and ``D`` (NAO, NAO) on a CUDA device; the
    shells, exponents and contraction coefficients come from ``basis`` (a
    TAOBasis).  The backward pass returns grad_out * dJ/dcoords and
    grad_out * J_pq (the Coulomb matrix, computed only when D needs a gradient).
    """

    _fn = None

    @classmethod
    def function(cls):
        if cls._fn is None:
            import torch

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, coords, D, basis, omega):
                    tb = with_coords(basis, coords.detach().cpu().numpy())
                    e, g, jm = _device_call(tb, D, omega, D.requires_grad)
                    ctx.save_for_backward(torch.as_tensor(g, dtype=coords.dtype, device=coords.device),
                                          jm if jm is not None else torch.empty(0, device=D.device))
                    ctx.want_jmat = jm is not None
                    return torch.tensor(e, dtype=torch.float64, device=D.device)

                @staticmethod
                def backward(ctx, grad_out):
                    g, jm = ctx.saved_tensors
                    gc = grad_out.to(g.device) * g
                    gd = grad_out * jm if ctx.want_jmat else None
                    return gc, gd, None, None

            cls._fn = _Fn
        return cls._fn


def coulomb_energy(coords, D, basis, omega: float = 0.0):
    """J as a differentiable function of the atom coordinates and the density."""
    return CoulombEnergy.function().apply(coords, D, basis, omega)
