"""CUDA-graph SCF iterations against eager ones: the same kernels in the same
order, so the converged energy and iteration count agree (bit-level for FP64
K with full eigensolves; to the refinement tolerance with the device-side
refinement loop)."""
import numpy as np
import pytest

import tinyscf
from conftest import BAS, DFBAS, xyz

pytestmark = pytest.mark.gpu


def solve(name, kmode, dmode, graph, ene_tol=1e-10):
    e = tinyscf.TinySCF(BAS, DFBAS, xyz(name), 60)
    e.setup()
    e.set_k_precision(kmode)
    e.set_density_solver(dmode)
    e.set_graph(graph)
    e.s.ene_tol = ene_tol
    c0 = e.counters()
    e.do_SCF()
    c1 = e.counters()
    out = dict(E=e.energy, it=e.s.iter, D=e.mat("D_mat"), F=e.mat("F_mat"), launches=c1[0] - c0[0],
               eig=c1[3] - c0[3], refine=c1[4] - c0[4], stats=e.timing_stats())
    e.free()
    return out


def test_graph_fp64_matches_eager():
    a = solve("c10h22", tinyscf.K_FP64, tinyscf.DENSITY_EIG, False)
    b = solve("c10h22", tinyscf.K_FP64, tinyscf.DENSITY_EIG, True)
    assert a["it"] == b["it"]
    assert abs(a["E"] - b["E"]) < 1e-11, (a["E"], b["E"])
    assert np.abs(a["D"] - b["D"]).max() < 1e-10
    # every iteration timed, graph launches included
    assert b["stats"]["ITER"][1] == b["it"]


@pytest.mark.parametrize("name", ["water", "c20h42"])
def test_graph_mixed_refine_matches_eager(name):
    a = solve(name, tinyscf.K_MIXED, tinyscf.DENSITY_REFINE, False)
    b = solve(name, tinyscf.K_MIXED, tinyscf.DENSITY_REFINE, True)
    assert abs(a["E"] - b["E"]) < 1e-9, (a["E"], b["E"])
    assert abs(a["it"] - b["it"]) <= 1
    assert b["refine"] > 0


def test_graph_reused_across_solves():
    e = tinyscf.TinySCF(BAS, DFBAS, xyz("c10h22"), 60)
    e.setup()
    e.set_k_precision(tinyscf.K_MIXED)
    e.set_density_solver(tinyscf.DENSITY_REFINE)
    e.set_graph(True)
    energies = []
    for _ in range(3):
        e.reset_scf()
        e.do_SCF()
        energies.append(e.energy)
    e.set_graph(False)
    e.reset_scf()
    e.do_SCF()
    energies.append(e.energy)
    e.free()
    assert max(energies) - min(energies) < 1e-9, energies
