"""ctypes wrapper of the CPU oracle (oracle/gci_oracle.c).

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA library.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU legs may use it.

The oracle takes a raw molecule (atom coordinates, shells with angular
momentum, exponents and unnormalised contraction coefficients), normalises
it with its own restatement of basis_NormalizeCntrCoeffs / SpherGTO_NormFactors
(src/basis/basis_sets.f90:894-945, src/basis/sphergto.f90:166-269) and runs
the FP64 restatement of the reference path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_i64 = C.c_int64
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)
_pl = C.POINTER(C.c_int64)


def build() -> Path:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


class _Basis(C.Structure):
    _fields_ = [("nshells", C.c_int), ("coords", _pd), ("L", _pi), ("nprim", _pi), ("prim_off", _pi),
                ("exps", _pd), ("coefs", _pd), ("T_off", _pi), ("T", _pd), ("spher", C.c_int)]


class _Chol(C.Structure):
    _fields_ = [("nao", _i64), ("nshellpairs", _i64), ("norbpairs", _i64), ("nvecs", _i64),
                ("npivshellpairs", _i64), ("nsubsets", _i64), ("max_subset_dim", _i64),
                ("converged", C.c_int), ("trace_error", C.c_double), ("dmax_final", C.c_double),
                ("shellpairs", _pi), ("shellpairloc", _pl), ("shellpairdim", _pi), ("subsetdim", _pl),
                ("subsetbounds", _pl), ("pivots", _pi), ("pivot_order", _pl), ("pivot_dmax", _pd),
                ("pivshellpairs", _pi), ("pivshellpairloc", _pl), ("pivshellpairdim", _pi),
                ("pivorbpairs", _pi), ("inv_l", _pd), ("rkpq", _pd), ("n_macro", _i64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.orc_boys_init.argtypes = [C.c_int]
        L.orc_fm_reference.argtypes = [C.c_int, C.c_double]
        L.orc_fm_reference.restype = C.c_double
        L.orc_fm_batch.argtypes = [C.c_int, _i64, _pd, _pd]
        L.orc_spher_u.argtypes = [C.c_int, _pd]
        L.orc_normalize_cntr.argtypes = [C.c_int, C.c_int, _pi, _pi, _pd, _pd, _pd, C.c_int]
        L.orc_spher_norms.argtypes = [C.c_int, C.c_int, _pi, _pi, _pd, _pd, _pd, C.c_int]
        L.orc_eri_quartet.argtypes = [C.POINTER(_Basis), C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _pd]
        L.orc_cholesky.argtypes = [C.POINTER(_Basis), C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.POINTER(_Chol)]
        L.orc_cholesky_forced.argtypes = [C.POINTER(_Basis), C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                          C.c_int, _pl, _i64, C.c_int, C.POINTER(_Chol)]
        L.orc_stats.argtypes = [_pd, C.c_int]
        L.orc_stats_reset.argtypes = []
        L.orc_rtuv.argtypes = [C.c_int, _pd, C.c_double, C.c_double, C.c_double, C.c_double, _pd]
        L.orc_et_coeffs.argtypes = [C.c_int, C.c_double, C.c_double, _pd]
        L.orc_eri_quartets_batch.argtypes = [C.POINTER(_Basis), _i64, _pi, C.c_double, C.c_int]
        L.orc_eri_quartets_batch.restype = C.c_double
        L.orc_set_eri_scheme.argtypes = [C.c_int]
        L.orc_set_eri_scheme.restype = None
        L.orc_chol_free.argtypes = [C.POINTER(_Chol)]
        L.orc_mo_transf.argtypes = [C.POINTER(_Chol), C.POINTER(_Basis), _pi, _pd, _i64, _i64, _i64, _pd, _i64,
                                    _i64, _i64, C.c_int, _pd]
        L.orc_eri_full.argtypes = [C.POINTER(_Basis), _pi, _i64, C.c_double, C.c_int, _pd]
        L.orc_coulomb_energy_grad.argtypes = [C.POINTER(_Basis), _pi, C.c_int, _pi, _pd, _i64, C.c_double, C.c_int,
                                              _pd, _pd]
        if L.orc_boys_init(20) != 0:
            raise RuntimeError("orc_boys_init failed")
        _lib = L
    return _lib


def _p(a, t=_pd):
    return a.ctypes.data_as(t)


def ncart(l):
    return (l + 1) * (l + 2) // 2


def fm_reference(m: int, x: float) -> float:
    return lib().orc_fm_reference(m, float(x))


def boys(m: int, x) -> np.ndarray:
    x = np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.float64)))
    out = np.empty((x.size, m + 1))
    lib().orc_fm_batch(m, x.size, _p(x), _p(out))
    return out


def spher_u(L: int) -> np.ndarray:
    U = np.zeros((2 * L + 1, ncart(L)))
    lib().orc_spher_u(L, _p(U))
    return U


@dataclass
class OracleBasis:
    """Per-shell arrays of a normalised basis as the oracle consumes them."""
    L: np.ndarray
    nprim: np.ndarray
    prim_off: np.ndarray
    exps: np.ndarray
    coefs: np.ndarray
    coords: np.ndarray          # (nshells, 3)
    T_off: np.ndarray
    T: np.ndarray
    spher: int
    shell_atom: np.ndarray
    shell_loc: np.ndarray
    nao: int
    natoms: int
    _keep: list = field(default_factory=list)

    def cstruct(self) -> _Basis:
        b = _Basis(len(self.L), _p(self.coords), _p(self.L, _pi), _p(self.nprim, _pi), _p(self.prim_off, _pi),
                   _p(self.exps), _p(self.coefs), _p(self.T_off, _pi), _p(self.T), int(self.spher))
        return b


def make_basis(atoms, shells, spher: bool = True) -> OracleBasis:
    """atoms: (natoms, 3) coordinates in bohr; shells: list of (atom, L, exps, raw_coefs)."""
    atoms = np.asarray(atoms, dtype=np.float64)
    ns = len(shells)
    Ls = np.array([s[1] for s in shells], dtype=np.int32)
    npr = np.array([len(s[2]) for s in shells], dtype=np.int32)
    ld = int(npr.max())
    E = np.zeros((ns, ld))
    Cf = np.zeros((ns, ld))
    for i, s in enumerate(shells):
        E[i, :npr[i]] = s[2]
        Cf[i, :npr[i]] = s[3]
    E = np.ascontiguousarray(E)
    Cf = np.ascontiguousarray(Cf)
    ldc = ncart(int(Ls.max()))
    lds = 2 * int(Ls.max()) + 1
    ncart_n = np.zeros((ns, ldc))
    nsph = np.zeros((ns, lds))
    L = lib()
    L.orc_normalize_cntr(ns, ld, _p(Ls, _pi), _p(npr, _pi), _p(E), _p(Cf), _p(ncart_n), ldc)
    L.orc_spher_norms(ns, ld, _p(Ls, _pi), _p(npr, _pi), _p(E), _p(Cf), _p(nsph), lds)
    prim_off = np.zeros(ns, dtype=np.int32)
    exps, coefs, T, T_off = [], [], [], np.zeros(ns, dtype=np.int32)
    off = 0
    toff = 0
    nf = []
    for i in range(ns):
        prim_off[i] = off
        exps.extend(E[i, :npr[i]])
        coefs.extend(Cf[i, :npr[i]])
        off += npr[i]
        l = int(Ls[i])
        if spher:
            M = nsph[i, :2 * l + 1, None] * spher_u(l)
        else:
            M = np.diag(ncart_n[i, :ncart(l)])
        T_off[i] = toff
        T.extend(M.ravel())
        toff += M.size
        nf.append(M.shape[0])
    shell_atom = np.array([s[0] for s in shells], dtype=np.int32)
    loc = np.concatenate([[0], np.cumsum(nf)[:-1]]).astype(np.int32)
    return OracleBasis(L=Ls, nprim=npr, prim_off=prim_off, exps=np.array(exps), coefs=np.array(coefs),
                       coords=np.ascontiguousarray(atoms[shell_atom]), T_off=T_off, T=np.array(T),
                       spher=int(spher), shell_atom=shell_atom, shell_loc=loc, nao=int(sum(nf)),
                       natoms=len(atoms))


def eri_quartet(b: OracleBasis, A, B, Cc, D, kappa=0.0) -> np.ndarray:
    nf = [(2 * int(b.L[s]) + 1) if b.spher else ncart(int(b.L[s])) for s in (A, B, Cc, D)]
    out = np.zeros(int(np.prod(nf)))
    bs = b.cstruct()
    rc = lib().orc_eri_quartet(C.byref(bs), A, B, Cc, D, kappa, _p(out))
    if rc != 0:
        raise RuntimeError(f"orc_eri_quartet failed ({rc})")
    return out.reshape(nf[::-1]).transpose(3, 2, 1, 0)   # [a, b, c, d]


def herm_idx(t: int, u: int, v: int) -> int:
    """Level-major position of the Hermite index (t, u, v) (all of level < t+u+v first)."""
    n = t + u + v
    return n * (n + 1) * (n + 2) // 6 + (u + v) * (u + v + 1) // 2 + v


def rtuv(n: int, F, alpha: float, X: float, Y: float, Z: float) -> np.ndarray:
    """R_tuv for t+u+v <= n (level-major order) from F_0..F_n."""
    Fv = np.ascontiguousarray(F, dtype=np.float64)
    out = np.zeros((n + 1) * (n + 2) * (n + 3) // 6)
    lib().orc_rtuv(n, _p(Fv), alpha, X, Y, Z, _p(out))
    return out


def et_coeffs(emax: int, p: float, X: float) -> np.ndarray:
    """Single-centre Hermite coefficients E^{e}_t, shape (emax+1, emax+1)."""
    out = np.zeros((emax + 1) * (emax + 1))
    lib().orc_et_coeffs(emax, p, X, _p(out))
    return out.reshape(emax + 1, emax + 1)


def eri_quartets_batch(b: OracleBasis, quads, kappa=0.0, nthreads=0) -> float:
    """Evaluate the shell quartets `quads` (n x 4, 0-based) over nthreads OpenMP
    threads and return the sum of the integrals (timing samples)."""
    q = np.ascontiguousarray(np.asarray(quads, dtype=np.int32).reshape(-1, 4))
    return float(lib().orc_eri_quartets_batch(C.byref(b.cstruct()), q.shape[0], _p(q, _pi), kappa, nthreads))


def eri_full(b: OracleBasis, kappa=0.0, nthreads=0) -> np.ndarray:
    n = b.nao
    out = np.zeros(n ** 4)
    bs = b.cstruct()
    loc = b.shell_loc.astype(np.int32)
    rc = lib().orc_eri_full(C.byref(bs), _p(loc, _pi), n, kappa, nthreads, _p(out))
    if rc != 0:
        raise RuntimeError(f"orc_eri_full failed ({rc})")
    return out.reshape(n, n, n, n, order="F")   # [p, q, r, s]


def _arr(ptr, n, dtype):
    if n <= 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype).copy()


@dataclass
class OracleCholesky:
    nao: int
    nvecs: int
    norbpairs: int
    nshellpairs: int
    nsubsets: int
    max_subset_dim: int
    converged: bool
    trace_error: float
    n_macro: int
    shellpairs: np.ndarray       # (nsp, 2) 0-based shells (A >= B)
    shellpairloc: np.ndarray     # (nsp, 3) 0-based FULL, SUBSET_STORAGE, SUBSET_INDEX
    shellpairdim: np.ndarray
    subsetdim: np.ndarray
    subsetbounds: np.ndarray     # (nsubsets, 2) 0-based
    pivots: np.ndarray
    pivot_order: np.ndarray      # 0-based FULL index per selection
    pivot_dmax: np.ndarray
    pivshellpairs: np.ndarray
    pivshellpairloc: np.ndarray
    pivshellpairdim: np.ndarray
    pivorbpairs: np.ndarray
    inv_l: np.ndarray            # (nvecs, nvecs)
    rkpq: np.ndarray | None      # (nvecs, max_subset_dim, nsubsets)
    _raw: _Chol | None = None
    _basis: OracleBasis | None = None


def cholesky(b: OracleBasis, tau: float, kappa: float = 0.0, want_rkpq: bool = True,
             decode_storage: bool = False, nthreads: int = 0, max_block_dim: int = 4000,
             forced_order=None) -> OracleCholesky:
    """Two-step Cholesky; with ``forced_order`` (0-based FULL pivot indices) only step 2 runs."""
    res = _Chol()
    bs = b.cstruct()
    if forced_order is None:
        rc = lib().orc_cholesky(C.byref(bs), tau, kappa, max_block_dim, int(want_rkpq), int(decode_storage),
                                nthreads, C.byref(res))
    else:
        fo = np.ascontiguousarray(forced_order, dtype=np.int64)
        rc = lib().orc_cholesky_forced(C.byref(bs), tau, kappa, max_block_dim, int(want_rkpq), int(decode_storage),
                                       nthreads, _p(fo, _pl), fo.size, 0, C.byref(res))
    if rc != 0:
        lib().orc_chol_free(C.byref(res))
        raise RuntimeError(f"orc_cholesky failed ({rc})")
    n, nsp, npq, ns, msd = res.nvecs, res.nshellpairs, res.norbpairs, res.nsubsets, res.max_subset_dim
    npsp = res.npivshellpairs
    out = OracleCholesky(
        nao=res.nao, nvecs=n, norbpairs=npq, nshellpairs=nsp, nsubsets=ns, max_subset_dim=msd,
        converged=bool(res.converged), trace_error=res.trace_error, n_macro=res.n_macro,
        shellpairs=_arr(res.shellpairs, 2 * nsp, np.int64).reshape(nsp, 2),
        shellpairloc=_arr(res.shellpairloc, 3 * nsp, np.int64).reshape(nsp, 3),
        shellpairdim=_arr(res.shellpairdim, nsp, np.int64),
        subsetdim=_arr(res.subsetdim, ns, np.int64),
        subsetbounds=_arr(res.subsetbounds, 2 * ns, np.int64).reshape(ns, 2),
        pivots=_arr(res.pivots, npq, np.int64),
        pivot_order=_arr(res.pivot_order, n, np.int64),
        pivot_dmax=_arr(res.pivot_dmax, n, np.float64),
        pivshellpairs=_arr(res.pivshellpairs, npsp, np.int64),
        pivshellpairloc=_arr(res.pivshellpairloc, npsp, np.int64),
        pivshellpairdim=_arr(res.pivshellpairdim, npsp, np.int64),
        pivorbpairs=_arr(res.pivorbpairs, n, np.int64),
        inv_l=_arr(res.inv_l, n * n, np.float64).reshape(n, n, order="F"),
        rkpq=(_arr(res.rkpq, n * msd * ns, np.float64).reshape(n, msd, ns, order="F") if res.rkpq else None),
        _raw=res, _basis=b)
    return out


def stats_reset() -> None:
    lib().orc_stats_reset()


ERI_TWO_CENTRE, ERI_REFERENCE_HRR = 1, 0


def set_eri_scheme(scheme: int) -> None:
    """1: two-centre Hermite form (default, as the CUDA library); 0: the reference's W-matrix + HRR."""
    lib().orc_set_eri_scheme(int(scheme))


def stats() -> np.ndarray:
    """Work counters: [0..4] GEMM flops, [5..7] quartets / primitive quartets / integrals, then per
    class (bra pair type, ket pair type) over 21 x 21 pair types (l <= 5)."""
    out = np.zeros(8 + 3 * 21 * 21)
    lib().orc_stats(_p(out), out.size)
    return out


def cholesky_stage(b: OracleBasis, tau: float, stage: int, nthreads: int = 0) -> int:
    """Run the pipeline up to a stage (1: diagonal + screen, 2: first macro iteration)."""
    res = _Chol()
    bs = b.cstruct()
    rc = lib().orc_cholesky_forced(C.byref(bs), tau, 0.0, 4000, 0, 0, nthreads, None, 0, stage, C.byref(res))
    lib().orc_chol_free(C.byref(res))
    if rc < 0:
        raise RuntimeError(f"orc_cholesky stage failed ({rc})")
    return rc


def mo_transf(ch: OracleCholesky, b: OracleBasis, CA, a0, a1, CB, b0, b1, nthreads=0) -> np.ndarray:
    """Rkab (nvecs, NA*NB); a0..a1, b0..b1 are 0-based inclusive column ranges."""
    CA = np.asfortranarray(CA, dtype=np.float64)
    CB = np.asfortranarray(CB, dtype=np.float64)
    NA, NB = a1 - a0 + 1, b1 - b0 + 1
    out = np.zeros(ch.nvecs * NA * NB)
    bs = b.cstruct()
    loc = b.shell_loc.astype(np.int32)
    rc = lib().orc_mo_transf(C.byref(ch._raw), C.byref(bs), _p(loc, _pi), _p(CA), CA.shape[0], a0, a1, _p(CB),
                             CB.shape[0], b0, b1, nthreads, _p(out))
    if rc != 0:
        raise RuntimeError(f"orc_mo_transf failed ({rc})")
    return out.reshape(ch.nvecs, NA * NB, order="F")


def coulomb_energy_grad(b: OracleBasis, Dm, kappa=0.0, nthreads=0):
    Dm = np.asfortranarray(Dm, dtype=np.float64)
    grad = np.zeros(3 * b.natoms)
    e = C.c_double(0.0)
    bs = b.cstruct()
    loc = b.shell_loc.astype(np.int32)
    sa = b.shell_atom.astype(np.int32)
    rc = lib().orc_coulomb_energy_grad(C.byref(bs), _p(sa, _pi), b.natoms, _p(loc, _pi), _p(Dm), b.nao, kappa,
                                       nthreads, C.byref(e), _p(grad))
    if rc != 0:
        raise RuntimeError(f"orc_coulomb_energy_grad failed ({rc})")
    return e.value, grad.reshape(b.natoms, 3)


def reconstruct_pq_rs(ch: OracleCholesky) -> np.ndarray:
    """(pq|rs) ~ sum_k R_kpq R_krs over the stored orbital pairs (FULL order)."""
    R = full_order_vectors(ch)
    return R.T @ R


def full_order_vectors(ch: OracleCholesky) -> np.ndarray:
    """Cholesky vectors (nvecs, norbpairs) with columns in the FULL storage order."""
    R = np.zeros((ch.nvecs, ch.norbpairs))
    for s in range(ch.nshellpairs):
        full, sub, X = ch.shellpairloc[s]
        d = ch.shellpairdim[s]
        R[:, full:full + d] = ch.rkpq[:, sub:sub + d, X]
    return R


def free(ch: OracleCholesky) -> None:
    if ch._raw is not None:
        lib().orc_chol_free(C.byref(ch._raw))
        ch._raw = None
