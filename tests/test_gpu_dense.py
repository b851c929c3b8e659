"""GPU tests of the FP64 dense kernels (dense_fp64.cu, DMMA tensor cores):
gci_dgemm against torch FP64 products, gci_cholesky_inverse (dpotrf + dtrtri
of real_linalg.f90:39-72) against numpy's Cholesky factor and the identity,
and gci_trsm_rlt (the pivot-batch solve of TwoStepCholesky_Step1.f90:859-881)
against a dense solve.

Tolerances: FP64 products agree to 1e-13 k max|A| max|B| per element
(summation order differs from torch's); the factor of a matrix with
condition number kappa agrees to ~kappa eps."""
import ctypes as C

import numpy as np
import pytest

from gammcor_integrals_b200 import _capi

pytestmark = pytest.mark.gpu


def _vp(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("m,n,k,alpha,beta", [(1, 1, 1, 1.0, 0.0), (128, 128, 16, 1.0, 0.0),
                                              (300, 200, 150, -1.0, 1.0), (129, 257, 33, 0.5, -2.0),
                                              (1000, 37, 2001, 1.0, 0.0), (5, 3000, 700, 1.0, 1.0),
                                              (64, 64, 0, 1.0, 0.5)])
def test_dgemm_matches_torch(gpu_lib, m, n, k, alpha, beta):
    import torch
    g = torch.Generator(device="cuda").manual_seed(m + 3 * n + 11 * k)
    lda, ldb, ldc = m + 3, n + 1, m + 5   # odd leading dimensions: unaligned columns
    Ab = torch.randn(max(k, 1), lda, dtype=torch.float64, device="cuda", generator=g)
    Bb = torch.randn(max(k, 1), ldb, dtype=torch.float64, device="cuda", generator=g)
    Cb = torch.randn(n, ldc, dtype=torch.float64, device="cuda", generator=g)
    A, B = Ab[:k, :m].T, Bb[:k, :n].T          # m x k, n x k column-major views
    ref = alpha * (A @ B.T) + beta * Cb[:, :m].T
    pad = Cb[:, m:].clone()
    torch.cuda.synchronize()
    _capi.check(gpu_lib.gci_dgemm(m, n, k, alpha, _vp(Ab), lda, _vp(Bb), ldb, beta, _vp(Cb), ldc))
    got = Cb[:, :m].T
    bound = 1e-13 * max(k, 1) * float(A.abs().max() if k else 0) * float(B.abs().max() if k else 0) + \
        1e-15 * ref.abs() + 1e-300
    assert bool(((got - ref).abs() <= bound).all()), float((got - ref).abs().max())
    assert torch.equal(Cb[:, m:], pad)   # nothing outside the m x n block is written


def _spd(n, seed, cond=1e6):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = np.logspace(0, -np.log10(cond), n)
    A = (Q * ev) @ Q.T
    return 0.5 * (A + A.T)


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 130, 257, 1000, 2500])
def test_cholesky_inverse(gpu_lib, n):
    import torch
    cond = 1e6
    A = _spd(n, n, cond=cond)
    At = torch.tensor(A.T.copy(), device="cuda")   # row r of At = column r of A (column-major A)
    Xt = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()   # the library's stream does not wait for torch's
    _capi.check(gpu_lib.gci_cholesky_inverse(n, _vp(At), n, _vp(Xt)))
    L = np.tril(At.T.cpu().numpy())
    X = Xt.T.cpu().numpy()
    Lref = np.linalg.cholesky(A)
    eps, nn = np.finfo(float).eps, max(n, 16)
    # both factors are backward stable: they differ by at most ~kappa(A) eps |L|
    assert np.abs(L - Lref).max() <= 50 * eps * cond * np.abs(Lref).max()
    assert np.all(np.triu(X, 1) == 0.0)
    assert np.abs(X @ L - np.eye(n)).max() <= nn * eps * cond
    Xref = np.linalg.inv(Lref)
    assert np.abs(X - Xref).max() <= nn * eps * cond * np.abs(Xref).max()


def test_cholesky_inverse_not_spd(gpu_lib):
    import torch
    n = 200
    A = _spd(n, 5, cond=10.0)
    A[150, 150] = -1.0   # leading minor of order 151 is indefinite
    At = torch.tensor(A.T.copy(), device="cuda")
    Xt = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = gpu_lib.gci_cholesky_inverse(n, _vp(At), n, _vp(Xt))
    assert rc == -5, rc   # GCI_ERR_NOT_SPD
    assert b"Cholesky factorization failed" in gpu_lib.gci_last_error()


@pytest.mark.parametrize("rows,w", [(1, 1), (1000, 31), (777, 32), (1000, 33), (5000, 100), (20000, 500)])
def test_trsm_rlt(gpu_lib, rows, w):
    import torch
    rng = np.random.default_rng(rows + w)
    Lp = np.linalg.cholesky(_spd(w, w + 1, cond=1e4))
    B = rng.standard_normal((rows, w))
    ref = np.linalg.solve(Lp, B.T).T          # X Lp^T = B
    Bt = torch.tensor(B.T.copy(), device="cuda")   # column-major rows x w
    Lt = torch.tensor(Lp.T.copy(), device="cuda")
    torch.cuda.synchronize()
    _capi.check(gpu_lib.gci_trsm_rlt(rows, w, _vp(Bt), rows, _vp(Lt), w))
    got = Bt.T.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-13 * 1e2 * max(w, 16) * np.abs(ref).max()
