"""Failure paths of the engine, exercised without faulting the GPU.

* SCF divergence guard: a density full of NaN, injected from the host through
  TinySCF_set_density, makes the first energy non-finite; the solve restarts
  from the SAD guess once (counter [6]) and ends at the reference's energy
  with the reference's iteration count (the reference has no guard: its loop,
  TinySCF.c:386-429, would carry the NaN to the end)."""
import os

import numpy as np
import pytest

import tinyscf
from conftest import BAS, DFBAS, GOLDEN, xyz

pytestmark = pytest.mark.gpu


def test_nan_density_restarts_from_sad():
    gold = np.load(os.path.join(GOLDEN, "water_ref.npz"))
    e = tinyscf.TinySCF(BAS, DFBAS, xyz("water"), 30)
    e.setup()
    n, o = e.s.nbasfuncs, e.s.n_occ
    e.set_density(np.full((n, n), np.nan), np.full((n, o), np.nan))
    e.do_SCF()
    assert e.counters()[6] == 1
    assert abs(e.energy - float(gold["energies"][-1])) < 1e-9
    assert e.s.iter == len(gold["energies"])
    e.free()


def test_guard_stays_off_on_a_normal_solve():
    e = tinyscf.TinySCF(BAS, DFBAS, xyz("c10h22"), 30)
    e.setup()
    e.do_SCF()
    assert e.counters()[6] == 0
    e.free()
