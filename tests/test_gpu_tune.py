"""Autotuner: every candidate computes the same values (the FFMA tile shapes
bit for bit, the FP64 tensor-core tiles to rounding), so a tuned engine
reproduces an untuned one; the tuned knobs show up in the tuner's table."""
import numpy as np
import pytest

import tinyscf
from conftest import BAS, DFBAS, xyz

pytestmark = pytest.mark.gpu


def _solve(name):
    """K of one Fock build on the SAD density, then a full SCF from it."""
    e = tinyscf.TinySCF(BAS, DFBAS, xyz(name), 60)
    e.setup()
    e.s.iter = 0
    e.build_FockMat()
    K = e.mat("K_mat")
    e.reset_scf()
    e.s.ene_tol = 1e-10
    e.do_SCF()
    out = (e.energy, e.s.iter, K, e.df_tensor())
    e.free()
    return out


def test_tuned_engine_matches_untuned():
    """The tuned candidates round differently from the untuned defaults only in
    the last bits: the same K from the same density to 1e-10, the same DF
    tensor to 1e-13 relative, and SCFs that converge to the same energy (an
    iteration more or less where the 1e-10 threshold is crossed)."""
    tinyscf.set_autotune(False)
    try:
        E0, it0, K0, B0 = _solve("c10h22")
    finally:
        tinyscf.set_autotune(True)
    E1, it1, K1, B1 = _solve("c10h22")
    assert abs(it0 - it1) <= 1, (it0, it1)
    assert abs(E0 - E1) < 1e-9, (E0, E1)
    assert np.abs(K0 - K1).max() < 1e-10
    assert np.abs(B0 - B1).max() < 1e-13 * max(1.0, np.abs(B0).max())
    rep = tinyscf.autotune_report()
    for key in ("3c:", "dgemm:", "ksyrk:", "khalf:", "jrows:"):
        assert key in rep, rep


_PINNED = r"""
import sys
import numpy as np
import tinyscf
from conftest import BAS, DFBAS
e = tinyscf.TinySCF(BAS, DFBAS, sys.argv[2], 60)
e.setup()
e.s.iter = 0
e.build_FockMat()
np.save(sys.argv[1], e.mat("K_mat"))
e.free()
print(tinyscf.autotune_report())
"""


@pytest.mark.parametrize("name", ["c10h22", "hcn"])
def test_pinned_half_transform_variants_match(tmp_path, name):
    """Each exchange half-transform variant (64x64 FFMA, 64x256 FFMA, 64x256
    DMMA, pipelined persistent DMMA), pinned through TINYSCF_TUNE_FILE in a
    fresh process, builds the tuned engine's K from the same (SAD) density up
    to summation-order rounding. C10H22 has an even number of aux functions (16-byte row copies
    in the pipelined kernel), HCN an odd one (8-byte copies)."""
    import os
    import subprocess
    import sys
    if name == "hcn":
        path = tmp_path / "hcn.xyz"
        path.write_text("3\n0\nH 0.0 0.0 -1.066\nC 0.0 0.0 0.0\nN 0.0 0.0 1.156\n")
        path = str(path)
    else:
        path = xyz(name)
    e = tinyscf.TinySCF(BAS, DFBAS, path, 60)
    e.setup()
    e.s.iter = 0
    e.build_FockMat()
    K = e.mat("K_mat")
    nbf, nocc, naux = e.s.nbasfuncs, e.s.n_occ, e.s.df_nbf
    e.free()
    assert (naux % 2 == 0) == (name == "c10h22")
    keys = [line.split()[0] for line in tinyscf.autotune_report().splitlines()
            if line.startswith("khalf:%d:%d:%d:" % (nbf, nocc, naux))]
    assert len(keys) == 1, keys
    here = os.path.dirname(os.path.abspath(__file__))
    for variant in (0, 1, 2, 3):
        tune = tmp_path / ("tune%d.txt" % variant)
        tune.write_text("%s %d 0.0\n" % (keys[0], variant))
        out = tmp_path / ("K%d.npy" % variant)
        env = dict(os.environ, TINYSCF_TUNE_FILE=str(tune),
                   PYTHONPATH=os.pathsep.join([here, os.path.join(os.path.dirname(here), "yatscf-df_b200"),
                                               os.environ.get("PYTHONPATH", "")]))
        res = subprocess.run([sys.executable, "-c", _PINNED, str(out), path], env=env, capture_output=True,
                             text=True, timeout=600)
        assert res.returncode == 0, res.stderr[-2000:]
        assert "%s -> %d" % (keys[0], variant) in res.stdout, res.stdout
        # summation order differs between the FFMA and DMMA tiles: a few 1e-12
        # on C10H22; the parity tests hold K to 1e-10 against the golden files
        assert np.abs(np.load(out) - K).max() < 1e-10, variant


_PINNED_FAST = r"""
import sys
import numpy as np
import tinyscf
from conftest import BAS, DFBAS, xyz
e = tinyscf.TinySCF(BAS, DFBAS, xyz("c10h22"), 60)
e.setup()
e.set_k_precision(tinyscf.K_MIXED)
e.set_density_solver(tinyscf.DENSITY_REFINE)
e.set_graph(True)
e.set_guess(tinyscf.GUESS_LEARNED)
e.reset_scf()
e.s.ene_tol = 1e-9
e.do_SCF()
np.save(sys.argv[1], np.array([e.energy, e.s.iter]))
np.save(sys.argv[2], e.mat("D_mat"))
e.free()
print(tinyscf.autotune_report())
"""


def test_pinned_dgemm_variants_match(tmp_path):
    """The accelerated form (learned guess, tensor-core K, subspace refinement,
    CUDA graph) with every tuned FP64 GEMM shape pinned to one tile variant
    (TINYSCF_TUNE_FILE, fresh process): 64x64 FFMA, 128x128 / 64x64 DMMA and
    the 32x32 DMMA tile with K split over warps all reach the same energy and
    density."""
    import os
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    env0 = dict(os.environ, PYTHONPATH=os.pathsep.join([here, os.path.join(os.path.dirname(here), "yatscf-df_b200"),
                                                         os.environ.get("PYTHONPATH", "")]))
    out = {}
    keys = None
    for variant in (None, 0, 3, 4, 5):
        tune = tmp_path / ("tune%s.txt" % variant)
        if variant is not None:
            tune.write_text("".join("%s %d 0.0\n" % (k, variant) for k in keys))
        e_out, d_out = tmp_path / ("E%s.npy" % variant), tmp_path / ("D%s.npy" % variant)
        res = subprocess.run([sys.executable, "-c", _PINNED_FAST, str(e_out), str(d_out)],
                             env=dict(env0, TINYSCF_TUNE_FILE=str(tune)), capture_output=True, text=True, timeout=600)
        assert res.returncode == 0, res.stderr[-2000:]
        if variant is None:
            keys = [line.split()[0] for line in res.stdout.splitlines() if line.startswith("dgemm:")]
            assert len(keys) >= 5, res.stdout
        else:
            for k in keys:
                assert "%s -> %d" % (k, variant) in res.stdout, (k, variant)
        out[variant] = (np.load(e_out), np.load(d_out))
    E0, D0 = out[None]
    for variant in (0, 3, 4, 5):
        E, D = out[variant]
        # converged to 1e-9 Eh from slightly different rounding: the energies
        # agree to the convergence threshold, the densities to its square root
        assert abs(E[0] - E0[0]) < 1e-8, (variant, E, E0)
        assert np.abs(D - D0).max() < 1e-4, variant
