"""The engine's FP64 symmetric eigensolver (Householder tridiagonalisation,
divide and conquer, WY back-transformation; the device replacement of the
reference's LAPACKE_dsyev at TinySCF.c:65, build_DF_tensor.c:217 and
build_density.c:54) through the C ABI, against LAPACK (numpy) on the same
matrices.

Tolerances, relative to max|A|: eigenvalues within 1e-12 of LAPACK's,
residual max|V A - diag(w) V| and orthogonality max|V V^T - I| below
1e-12 (both methods are backward stable: their errors are a few n eps)."""
import numpy as np
import pytest

import tinyscf

pytestmark = pytest.mark.gpu


def _check(A, tol=1e-12):
    n = A.shape[0]
    w, V = tinyscf.eigh(A)
    scale = max(np.abs(A).max(), 1e-300)
    ref = np.linalg.eigvalsh(A)
    assert np.all(np.diff(w) >= 0)
    assert np.abs(w - ref).max() / scale < tol
    assert np.abs(V @ A - w[:, None] * V).max() / scale < tol
    assert np.abs(V @ V.T - np.eye(n)).max() < tol
    return w, V


@pytest.mark.parametrize("n", [1, 2, 3, 5, 31, 32, 33, 64, 100, 257, 1010])
def test_random_symmetric(n):
    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, n))
    _check(X + X.T)


def test_clustered_spectrum():
    """Near-degenerate clusters (the core orbitals of a long alkane): deflation by close pairs."""
    rng = np.random.default_rng(7)
    n = 400
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    w = np.r_[np.full(40, -11.2) + 1e-10 * rng.standard_normal(40), np.full(30, -0.5), np.linspace(-1, 3, n - 70)]
    _check((Q * w) @ Q.T)


def test_ill_conditioned_metric_inverse_sqrt():
    """Spectrum of the C40H82 DF metric (4.5e-8 .. 2.8e3): X = V^T w^-1/2 V
    satisfies X A X = I to the conditioning, as LAPACK's does."""
    rng = np.random.default_rng(11)
    n = 600
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    w = np.logspace(np.log10(4.5e-8), np.log10(2.8e3), n)
    A = (Q * w) @ Q.T
    A = 0.5 * (A + A.T)
    wg, V = _check(A)
    X = V.T @ (V / np.sqrt(wg)[:, None])
    wl, Vl = np.linalg.eigh(A)
    Xl = Vl @ (Vl.T / np.sqrt(wl)[:, None])
    err_g = np.abs(X @ A @ X - np.eye(n)).max()
    err_l = np.abs(Xl @ A @ Xl - np.eye(n)).max()
    assert err_g < 10 * max(err_l, 1e-10)


@pytest.mark.parametrize("kind", ["identity", "diag_repeated", "wilkinson", "zero", "tridiagonal_split"])
def test_structured(kind):
    if kind == "identity":
        A = 3.0 * np.eye(50)
    elif kind == "diag_repeated":
        A = np.diag(np.r_[np.ones(10), 2.0 * np.ones(10), -np.ones(5)])
    elif kind == "wilkinson":
        A = np.diag(np.abs(np.arange(-10, 11)).astype(float)) + np.diag(np.ones(20), 1) + np.diag(np.ones(20), -1)
    elif kind == "zero":
        A = np.zeros((17, 17))
    else:   # exact zeros on the off-diagonal: independent blocks
        A = np.diag(np.arange(40, dtype=float))
        A[5, 6] = A[6, 5] = 0.3
        A[20, 21] = A[21, 20] = -0.7
    _check(A)


def test_engine_eigensolves_match_lapack():
    """X = S^-1/2 of a real molecule (C10H22) from the engine's eigensolver
    against X from LAPACK on the engine's own S."""
    from conftest import BAS, DFBAS, xyz
    e = tinyscf.TinySCF(BAS, DFBAS, xyz("c10h22"), 30)
    e.setup()
    S, X = e.mat("S_mat"), e.mat("X_mat")
    w, V = np.linalg.eigh(S)
    Xl = (V / np.sqrt(w)) @ V.T
    assert np.abs(X - Xl).max() < 1e-10 * np.abs(Xl).max()
    e.free()
