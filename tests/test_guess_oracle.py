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
