"""The recursions of csrc/dense_fp64.cu restated step by step in numpy, on CPU:
the same split rule, the same four products per level (with the zero parts of
the triangular operands left out exactly as the GEMM flags leave them out)
and the same use of the upper triangle as scratch.  This checks the algebra
of the drivers (real_Cholesky + real_LowerTriangularInverse of
real_linalg.f90:39-72, and the pivot-batch solve of
TwoStepCholesky_Step1.f90:859-881) independently of the GPU; the kernels
themselves are checked in tests/test_gpu_dense.py."""
import numpy as np
import pytest
from scipy.linalg import solve_triangular

LEAF, TRSM_W = 64, 32


def _potrf_rec(a, x, off, n):
    if n <= LEAF:
        L = np.linalg.cholesky(np.tril(a[off:off + n, off:off + n]) + np.tril(a[off:off + n, off:off + n], -1).T)
        a[off:off + n, off:off + n] = np.where(np.tri(n, dtype=bool), L, a[off:off + n, off:off + n])
        # the leaf kernel's inverse: column by column substitution (exact zeros above the diagonal)
        x[off:off + n, off:off + n] = solve_triangular(L, np.eye(n), lower=True)
        return
    n1 = (n // 2 + LEAF - 1) // LEAF * LEAF
    n2, o2 = n - n1, off + n1
    _potrf_rec(a, x, off, n1)
    X11 = np.tril(x[off:o2, off:o2])
    x[o2:off + n, off:o2] = a[o2:off + n, off:o2] @ X11.T          # L21 = A21 X11^T (held in X21)
    L21 = x[o2:off + n, off:o2].copy()
    a[o2:off + n, o2:off + n] -= np.tril(L21 @ L21.T)              # lower tiles of A22 -= L21 L21^T
    _potrf_rec(a, x, o2, n2)
    a[o2:off + n, off:o2] = L21                                   # L21 into place
    a[off:o2, o2:off + n] = (L21 @ X11).T                         # T = L21 X11, transposed into A12
    x[o2:off + n, off:o2] = -np.tril(x[o2:off + n, o2:off + n]) @ a[off:o2, o2:off + n].T


def _trsm_rec(b, l, c0, w):
    if w <= TRSM_W:
        Lb = l[c0:c0 + w, c0:c0 + w]
        for j in range(w):                                          # substitution, one column at a time
            b[:, c0 + j] = (b[:, c0 + j] - b[:, c0:c0 + j] @ Lb[j, :j]) / Lb[j, j]
        return
    w1 = (w // 2 + TRSM_W - 1) // TRSM_W * TRSM_W
    _trsm_rec(b, l, c0, w1)
    b[:, c0 + w1:c0 + w] -= b[:, c0:c0 + w1] @ l[c0 + w1:c0 + w, c0:c0 + w1].T
    _trsm_rec(b, l, c0 + w1, w - w1)


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    m = (q * np.logspace(0, -4, n)) @ q.T
    return 0.5 * (m + m.T)


@pytest.mark.parametrize("n", [1, 64, 65, 129, 200, 300])
def test_recursive_cholesky_inverse(n):
    A = _spd(n, n)
    a, x = A.copy(), np.zeros_like(A)
    _potrf_rec(a, x, 0, n)
    L = np.tril(a)
    np.testing.assert_allclose(L, np.linalg.cholesky(A), atol=1e-10)
    np.testing.assert_allclose(x @ L, np.eye(n), atol=1e-9)
    assert np.all(np.triu(x, 1) == 0.0)


@pytest.mark.parametrize("w", [1, 32, 33, 70, 200])
def test_recursive_triangular_solve(w):
    rng = np.random.default_rng(w)
    Lp = np.linalg.cholesky(_spd(w, w + 3) + np.eye(w))
    B = rng.standard_normal((50, w))
    X = B.copy()
    _trsm_rec(X, Lp, 0, w)
    np.testing.assert_allclose(X @ Lp.T, B, atol=1e-10)
