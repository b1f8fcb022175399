"""Learned initial guess: the training kernels' gradients against the CPU
oracle, rotation invariance of the pair features and local target blocks,
and what the trained network gains over SAD on molecules it was not trained
on (same converged energy, fewer SCF iterations)."""
import os
import sys

import numpy as np
import pytest

import geometry
import tinyscf
from conftest import BAS, DFBAS, REPO, xyz

sys.path.insert(0, os.path.join(REPO, "oracle"))
import guess_oracle as go  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("din,hid,dout,n", [(16, 24, 10, 37), (128, 192, 75, 300), (128, 192, 225, 70)])
def test_mlp_gradient_matches_oracle(din, hid, dout, n):
    rng = np.random.default_rng(din + dout)
    p = rng.normal(scale=1.0 / np.sqrt(hid), size=go.param_count(din, hid, dout)).astype(np.float32)
    X = rng.normal(size=(n, din)).astype(np.float32)
    T = rng.normal(size=(n, dout)).astype(np.float32)
    loss, g = tinyscf.guess_mlp_grad(p, X, T, din, hid, dout)
    loss_ref, g_ref = go.loss_grad(p.astype(np.float64), X, T, din, hid, dout)
    assert abs(loss - loss_ref) < 1e-5 * abs(loss_ref)
    # FP32 kernels against the FP64 oracle
    assert np.abs(g - g_ref).max() < 1e-4 * np.abs(g_ref).max(), np.abs(g - g_ref).max()


def _dataset(atoms, tmp_path, name):
    path = str(tmp_path / (name + ".xyz"))
    geometry.write_xyz(path, atoms)
    e = tinyscf.TinySCF(BAS, DFBAS, path, 60)
    e.setup()
    e.s.ene_tol = 1e-11
    e.do_SCF()
    out = e.guess_dataset(e.mat("D_mat"))
    e.free()
    return out


def test_pair_features_and_blocks_are_rotation_invariant(tmp_path):
    atoms = geometry.water_cluster(3, nmax=4)
    xyz0 = np.array([a[1:] for a in atoms])
    q = np.array([0.3, -0.5, 0.7, 0.4])
    q /= np.linalg.norm(q)
    xyz1 = xyz0 @ geometry._rotation(q).T + np.array([1.0, -2.0, 0.5])
    rot = [(a[0], *map(float, r)) for a, r in zip(atoms, xyz1)]
    f0, t0, y0 = _dataset(atoms, tmp_path, "a")
    f1, t1, y1 = _dataset(rot, tmp_path, "b")
    assert (y0 == y1).all()
    assert np.abs(f0 - f1).max() < 1e-5
    # same density in the pair frames, to the SCF convergence
    assert np.abs(t0 - t1).max() < 1e-5, np.abs(t0 - t1).max()


def _solve(path, guess, ene_tol):
    e = tinyscf.TinySCF(BAS, DFBAS, path, 60)
    e.setup(guess=guess)
    e.s.ene_tol = ene_tol
    e.do_SCF()
    out = (e.energy, e.s.iter, e.guess_used())
    e.free()
    return out


@pytest.mark.skipif(not os.path.exists(tinyscf.GUESS_WEIGHTS), reason="no trained guess weights in the package")
def test_learned_guess_saves_iterations(tmp_path):
    """Against SAD (the reference's guess) and against SAD put through the same
    projection (what the network itself adds): same converged energy, fewer
    iterations, on water clusters (evaluation seeds 0-3, disjoint from the
    training seeds 10000+) and on C20H42 (longer than any training alkane)."""
    paths = []
    for seed in range(4):
        p = str(tmp_path / ("w%d.xyz" % seed))
        geometry.write_xyz(p, geometry.water_cluster(seed))
        paths.append(p)
    paths.append(xyz("c20h42"))
    its = {g: [] for g in (tinyscf.GUESS_SAD, tinyscf.GUESS_SAD_PROJECTED, tinyscf.GUESS_LEARNED)}
    for p in paths:
        E = {}
        for g in its:
            E[g], it, used = _solve(p, g, 1e-10)
            assert used == g
            its[g].append(it)
        assert abs(E[tinyscf.GUESS_LEARNED] - E[tinyscf.GUESS_SAD]) < 1e-8, (p, E)
        assert abs(E[tinyscf.GUESS_SAD_PROJECTED] - E[tinyscf.GUESS_SAD]) < 1e-8, (p, E)
    assert sum(its[tinyscf.GUESS_LEARNED]) < sum(its[tinyscf.GUESS_SAD_PROJECTED]) < sum(its[tinyscf.GUESS_SAD]), its
