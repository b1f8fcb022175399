"""The learned-guess MLP oracle against central finite differences, and the
host-side pair features / frames of the engine (no GPU needed)."""
import ctypes
import os
import sys

import numpy as np
import pytest

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


_EL = {"H": 0, "C": 5, "N": 6, "O": 7, "S": 15}
_BOHR = 1.0 / 0.52917720859


def _mol(atoms):
    el = [_EL[a[0]] for a in atoms]
    xyz = np.array([a[1:] for a in atoms], dtype=np.float64) * _BOHR
    am = [[0, 0, 1] if e == 0 else [0, 0, 0, 1, 1, 2] for e in el]
    return el, xyz, am


def _molecules():
    sys.path.insert(0, os.path.join(REPO, "yatscf-df_b200"))
    import geometry
    mols = {"water_cluster_%d" % s: geometry.water_cluster(s) for s in (0, 1, 2)}
    mols["propane"] = geometry.alkane(3)
    mols["hcn"] = [("H", 0.0, 0.0, -1.066), ("C", 0.0, 0.0, 0.0), ("N", 0.0, 0.0, 1.156)]
    mols["n2"] = [("N", 0.0, 0.0, 0.0), ("N", 0.0, 0.0, 1.10)]
    mols["oxygen_atom"] = [("O", 0.0, 0.0, 0.0)]
    # equal distances everywhere: the frame choice rests on the index tie-break
    mols["methane_td"] = [("C", 0.0, 0.0, 0.0), ("H", 0.63, 0.63, 0.63), ("H", -0.63, -0.63, 0.63),
                          ("H", -0.63, 0.63, -0.63), ("H", 0.63, -0.63, -0.63)]
    return mols


def test_pair_blocks_match_restatement():
    """The library's pair list, block types, local frames and features (host
    code, no GPU) against the scalar restatement: same blocks in the same
    order, frames to 1e-14, features equal after rounding to float32 (both
    evaluate the same double expressions; exp/cos may differ in the last
    double bit, which a float32 rounding almost never shows)."""
    sys.path.insert(0, os.path.join(REPO, "yatscf-df_b200"))
    import tinyscf
    for name, atoms in _molecules().items():
        el, xyz, am = _mol(atoms)
        ref = go.pair_blocks(el, xyz, am)
        lib = tinyscf.guess_pairs(el, xyz, am)
        assert len(ref) == len(lib["type"]), name
        assert np.array_equal(np.array([[r[0], r[1]] for r in ref]).reshape(-1, 2), lib["ab"]), name
        assert np.array_equal(np.array([r[2] for r in ref]), lib["type"]), name
        assert np.abs(np.array([r[3] for r in ref]) - lib["frame"]).max() < 1e-14, name
        f = np.array([r[4] for r in ref], dtype=np.float64).astype(np.float32)
        assert np.abs(f - lib["feat"]).max() <= 1e-7, name
        Q = lib["frame"]
        assert np.abs(np.einsum("kij,klj->kil", Q, Q) - np.eye(3)).max() < 1e-12, name   # orthonormal rows


def test_pair_features_invariant_under_rotation():
    """Rotating and translating the molecule leaves the blocks and features
    unchanged (to float32 rounding of coordinates) and rotates every frame:
    Q' = Q R^T for x' = R x + t."""
    sys.path.insert(0, os.path.join(REPO, "yatscf-df_b200"))
    import tinyscf
    rng = np.random.default_rng(11)
    for name in ("water_cluster_1", "propane", "hcn"):
        el, xyz, am = _mol(_molecules()[name])
        R = _random_rotation(rng)
        if np.linalg.det(R) < 0:
            R[:, 0] = -R[:, 0]
        a = tinyscf.guess_pairs(el, xyz, am)
        b = tinyscf.guess_pairs(el, xyz @ R.T + rng.normal(size=3), am)
        assert np.array_equal(a["ab"], b["ab"]) and np.array_equal(a["type"], b["type"]), name
        assert np.abs(a["feat"] - b["feat"]).max() < 1e-5, name
        if name != "hcn":   # a linear molecule's frames fall back to a fixed perpendicular
            assert np.abs(np.einsum("kij,lj->kil", a["frame"], R) - b["frame"]).max() < 1e-9, name


def test_pair_blocks_reject_uncovered_elements():
    sys.path.insert(0, os.path.join(REPO, "yatscf-df_b200"))
    import tinyscf
    el, xyz, am = _mol([("S", 0.0, 0.0, 0.0), ("H", 0.0, 0.0, 1.34)])
    assert go.pair_blocks(el, xyz, am) is None
    try:
        tinyscf.guess_pairs(el, xyz, am)
    except tinyscf.TinySCFError as err:
        assert "UNSUPPORTED" in str(err).upper(), err
    else:
        raise AssertionError("an uncovered element must be rejected")


def test_training_set_is_the_seeded_clusters_and_alkanes():
    """The trainer's molecules are fixed by their seeds: water clusters from
    seed 10000 on (4096 of them: seeds 10000-14095) and jittered alkanes from
    seed 20000 on, the same geometries on every call."""
    sys.path.insert(0, os.path.join(REPO, "yatscf-df_b200"))
    import geometry
    import guess_train
    jobs = guess_train.training_jobs(3, 2)
    assert [t for t, _ in jobs] == ["w10000", "w10001", "w10002", "a20000", "a20001"]
    assert jobs[1][1] == geometry.water_cluster(10001)
    again = guess_train.training_jobs(3, 2)
    assert all(a == b for (_, a), (_, b) in zip(jobs, again))
    for _, atoms in jobs[3:]:
        el = [a[0] for a in atoms]
        nc = el.count("C")
        assert 2 <= nc <= 10 and el.count("H") == 2 * nc + 2


def test_batched_generation_waves_with_fake_engines(monkeypatch, tmp_path):
    """guess_train.generate_batched on fake engines (host logic only): waves
    close when free memory drops below the reserve, largest molecules first,
    every engine is freed, unconverged molecules give no rows, and a failed
    set-up frees the engines of its wave."""
    sys.path.insert(0, os.path.join(REPO, "yatscf-df_b200"))
    import guess_train
    import tinyscf

    class S:
        def __init__(self):
            self.ene_tol, self.iter = 0.0, 0

    created, freed, waves = [], [], []

    class FakeEngine:
        def __init__(self, bas, dfbas, path, max_iter):
            self.path, self.max_iter, self.s = path, max_iter, S()
            created.append(self)

        def setup(self, guess=None):
            if "bad" in self.path:
                raise tinyscf.TinySCFError("setup")

        def mat(self, name):
            return np.zeros((2, 2))

        def guess_dataset(self, D):
            return np.ones((3, 4), np.float32), np.ones((3, 5), np.float32), np.zeros(3, np.int32)

        def free(self):
            freed.append(self)

    class FakeBatch:
        def __init__(self, engines):
            waves.append([len(open(e.path).read().splitlines()) for e in engines])
            for e in engines:
                e.s.iter = e.max_iter if "stuck" in e.path else 7

        def do_SCF(self):
            pass

        def free(self):
            pass

    free_mem = iter([50, 30, 50, 50, 30, 50, 50, 50] * 4)
    monkeypatch.setattr(tinyscf, "TinySCF", FakeEngine)
    monkeypatch.setattr(tinyscf, "TinySCFBatch", FakeBatch)
    monkeypatch.setattr(tinyscf, "load_library", lambda: None)
    monkeypatch.setattr(tinyscf, "set_autotune", lambda on: None)
    monkeypatch.setattr(tinyscf, "device_memory", lambda device=0: (next(free_mem) * 2 ** 30, 0))
    atoms = lambda n: [("H", 0.0, 0.0, float(k)) for k in range(n)]
    jobs = [("a", atoms(2)), ("stuck", atoms(5)), ("c", atoms(3)), ("d", atoms(4)), ("e", atoms(1))]
    f, t, y, iters, nw, unconv = guess_train.generate_batched(jobs, "b", "d", reserve_gb=40.0)
    assert nw == len(waves) == 2
    sizes = [n - 2 for w in waves for n in w]          # xyz lines minus the two header lines
    assert sizes == sorted(sizes, reverse=True)
    assert unconv == ["stuck"] and len(f) == len(iters) == 4 and all(i == 7 for i in iters)
    assert len(freed) == len(created) == 5

    created.clear(), freed.clear()
    with pytest.raises(tinyscf.TinySCFError):
        guess_train.generate_batched([("ok", atoms(3)), ("bad", atoms(2))], "b", "d", reserve_gb=0.0)
    assert len(freed) == len(created) == 2
