"""Autotuner: every candidate computes the same values (the FFMA tile shapes
bit for bit, the FP64 tensor-core tiles to rounding), so a tuned engine
reproduces an untuned one; the tuned knobs show up in the tuner's table."""
import numpy as np
import pytest

import tinyscf
from conftest import BAS, DFBAS, xyz

pytestmark = pytest.mark.gpu


def _solve(name):
    e = tinyscf.TinySCF(BAS, DFBAS, xyz(name), 60)
    e.setup()
    e.s.ene_tol = 1e-10
    e.do_SCF()
    out = (e.energy, e.s.iter, e.mat("K_mat"), e.df_tensor())
    e.free()
    return out


def test_tuned_engine_matches_untuned():
    tinyscf.set_autotune(False)
    try:
        E0, it0, K0, B0 = _solve("c10h22")
    finally:
        tinyscf.set_autotune(True)
    E1, it1, K1, B1 = _solve("c10h22")
    assert it0 == it1
    assert abs(E0 - E1) < 1e-10
    assert np.abs(K0 - K1).max() < 1e-11
    assert np.abs(B0 - B1).max() < 1e-13 * max(1.0, np.abs(B0).max())
    rep = tinyscf.autotune_report()
    for key in ("3c:", "dgemm:", "ksyrk:", "khalf:", "jrows:"):
        assert key in rep, rep
