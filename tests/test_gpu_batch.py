"""Batched SCF (one launch per phase over many molecules of uneven size)
against the same molecules solved one by one: the same iteration counts,
energies and densities."""
import numpy as np
import pytest

import geometry
import tinyscf
from conftest import BAS, DFBAS, xyz

pytestmark = pytest.mark.gpu


def _molecules(tmp_path):
    paths = [xyz("water"), xyz("c10h22")]
    for seed in range(4):
        p = str(tmp_path / ("w%d.xyz" % seed))
        geometry.write_xyz(p, geometry.water_cluster(seed, nmax=6))
        paths.append(p)
    # the same cluster twice (rotated): two members of one eigensolver group
    atoms = geometry.water_cluster(1, nmax=6)
    q = np.array([0.2, 0.9, -0.3, 0.1])
    q /= np.linalg.norm(q)
    rot = np.array([a[1:] for a in atoms]) @ geometry._rotation(q).T
    p = str(tmp_path / "w1r.xyz")
    geometry.write_xyz(p, [(a[0], *map(float, r)) for a, r in zip(atoms, rot)])
    paths.append(p)
    return paths


def _engine(p, guess=None, ene_tol=1e-10):
    e = tinyscf.TinySCF(BAS, DFBAS, p, 60)
    e.setup(guess=guess)
    e.s.ene_tol = ene_tol
    return e


@pytest.mark.parametrize("guess", [None, tinyscf.GUESS_LEARNED])
def test_batch_matches_single_molecule_scf(tmp_path, guess):
    paths = _molecules(tmp_path)
    single = []
    for p in paths:
        e = _engine(p, guess)
        e.do_SCF()
        single.append((e.energy, e.s.iter, e.mat("D_mat")))
        e.free()
    engines = [_engine(p, guess) for p in paths]
    b = tinyscf.TinySCFBatch(engines)
    b.do_SCF()
    ms, iters, launches = b.stats()
    for e, (E, it, D) in zip(engines, single):
        assert e.s.iter == it, (e.s.iter, it)
        assert abs(e.energy - E) < 1e-9, (e.energy, E)
        assert np.abs(e.mat("D_mat") - D).max() < 1e-8
    assert iters == max(s[1] for s in single)
    # phases are batched: far fewer launches than one solve per molecule would need
    assert launches < 80 * iters + 40 * len(paths), launches
    b.free()
    for e in engines:
        e.free()


def test_batch_mixed_k_matches_single_molecule(tmp_path):
    """Molecules set to the tensor-core incremental K iterate in the batch with
    the same final FP64 Fock build as their own SCF: same energies."""
    paths = _molecules(tmp_path)[:5]
    single = []
    for p in paths:
        e = _engine(p, tinyscf.GUESS_LEARNED)
        e.set_k_precision(tinyscf.K_MIXED)
        e.do_SCF()
        single.append((e.energy, e.s.iter))
        e.free()
    engines = []
    for p in paths:
        e = _engine(p, tinyscf.GUESS_LEARNED)
        e.set_k_precision(tinyscf.K_MIXED)
        engines.append(e)
    b = tinyscf.TinySCFBatch(engines)
    b.do_SCF()
    assert b.phase_ms()["FINAL"] > 0
    for e, (E, it) in zip(engines, single):
        assert abs(e.energy - E) < 1e-9, (e.energy, E)
        assert e.s.iter == it
    b.free()
    for e in engines:
        e.free()


def test_batch_mixed_k_one_launch_per_kernel(tmp_path, monkeypatch):
    """With TINYSCF_BATCH_KMIX=1 the mixed molecules' tensor-core K of a batch
    runs as one half-transform launch and one G GEMM launch over all of them:
    the same arithmetic per molecule as their builds one by one (identical
    energies and iteration counts), fewer launches."""
    paths = _molecules(tmp_path)[:6]
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("TINYSCF_BATCH_KMIX", mode)
        engines = []
        for p in paths:
            e = _engine(p, tinyscf.GUESS_LEARNED)
            e.set_k_precision(tinyscf.K_MIXED)
            engines.append(e)
        b = tinyscf.TinySCFBatch(engines)
        b.do_SCF()
        ms, iters, launches = b.stats()
        out[mode] = ([e.energy for e in engines], [e.s.iter for e in engines], launches)
        b.free()
        for e in engines:
            e.free()
    assert out["1"][0] == out["0"][0]
    assert out["1"][1] == out["0"][1]
    assert out["1"][2] < out["0"][2], (out["1"][2], out["0"][2])


def test_batch_refine_density_matches_single_molecule(tmp_path):
    """Molecules set to the subspace-refinement density solver refine in the
    batch as in their own SCF: same energies."""
    paths = _molecules(tmp_path)[:5]
    single = []
    for p in paths:
        e = _engine(p, tinyscf.GUESS_LEARNED)
        e.set_density_solver(tinyscf.DENSITY_REFINE)
        e.do_SCF()
        single.append((e.energy, e.s.iter))
        e.free()
    engines = []
    for p in paths:
        e = _engine(p, tinyscf.GUESS_LEARNED)
        e.set_density_solver(tinyscf.DENSITY_REFINE)
        engines.append(e)
    b = tinyscf.TinySCFBatch(engines)
    c0 = [e.counters() for e in engines]
    b.do_SCF()
    refined = sum(e.counters()[4] - c[4] for e, c in zip(engines, c0))
    for e, (E, it) in zip(engines, single):
        assert abs(e.energy - E) < 1e-9, (e.energy, E)
        assert abs(e.s.iter - it) <= 1
    assert refined > 0
    b.free()
    for e in engines:
        e.free()
