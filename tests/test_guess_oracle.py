"""The learned-guess MLP oracle against central finite differences, and the
host-side pair features / frames of the engine (no GPU needed)."""
import ctypes
import os
import sys

import numpy as np

from conftest import REPO

sys.path.insert(0, os.path.join(REPO, "oracle"))
import guess_oracle as go  # noqa: E402


def test_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    din, hid, dout, n = 7, 5, 4, 9
    p = rng.normal(scale=0.5, size=go.param_count(din, hid, dout))
    X = rng.normal(size=(n, din))
    T = rng.normal(size=(n, dout))
    loss, g = go.loss_grad(p, X, T, din, hid, dout)
    h = 1e-6
    fd = np.empty_like(p)
    for k in range(p.size):
        e = np.zeros_like(p)
        e[k] = h
        fd[k] = (go.loss_grad(p + e, X, T, din, hid, dout)[0] - go.loss_grad(p - e, X, T, din, hid, dout)[0]) / (2 * h)
    assert np.abs(fd - g).max() < 1e-8 * max(1.0, np.abs(g).max())
    assert loss > 0


def test_param_layout_sizes():
    assert go.param_count(128, 192, 225) == 128 * 192 + 192 + 192 * 192 + 192 + 192 * 225 + 225
    parts = go.split(np.arange(go.param_count(3, 2, 4), dtype=float), 3, 2, 4)
    assert [a.shape for a in parts] == [(3, 2), (2,), (2, 2), (2,), (2, 4), (4,)]


def _random_rotation(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    return q * np.sign(np.diag(r))


def _monomials(x, l):
    if l == 0:
        return np.ones(1)
    if l == 1:
        return x.copy()
    return np.array([x[a] * x[b] for a, b in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))])


def test_guess_rotation_transforms_cartesian_functions():
    """phi_m(x_m) = M phi_l(x_l) for x_m = Q^T x_l, shell by shell, and
    M(Q) M(Q^T) = I (the library's host code, no GPU needed)."""
    sys.path.insert(0, os.path.join(REPO, "yatscf-df_b200"))
    import tinyscf
    rng = np.random.default_rng(7)
    am = [0, 0, 0, 1, 1, 2]                     # cc-pVDZ heavy atom: s s s p p d
    for _ in range(5):
        Q = _random_rotation(rng)
        M = tinyscf.guess_rotation(am, Q)
        Mi = tinyscf.guess_rotation(am, Q.T)
        assert np.abs(M @ Mi - np.eye(len(M))).max() < 1e-12
        xl = rng.normal(size=3)
        xm = Q.T @ xl
        phi_l = np.concatenate([_monomials(xl, l) for l in am])
        phi_m = np.concatenate([_monomials(xm, l) for l in am])
        assert np.abs(phi_m - M @ phi_l).max() < 1e-12
