"""Mixed-precision exchange (tcgen05, split-BF16, incremental) against the
FP64 engine: first build within the split-BF16 error, increments whose error
shrinks with the density change, and the converged energy (after the final
FP64 Fock build) within 1e-8 Eh of the FP64 SCF."""
import numpy as np
import pytest

import tinyscf
from conftest import BAS, DFBAS, xyz

pytestmark = pytest.mark.gpu


def engine(name, mode, niters=60):
    e = tinyscf.TinySCF(BAS, DFBAS, xyz(name), niters)
    e.setup()
    e.set_k_precision(mode)
    return e


@pytest.mark.parametrize("name", ["water", "c10h22"])
def test_first_mixed_build_matches_fp64(name):
    ref = engine(name, tinyscf.K_FP64)
    ref.s.iter = 0
    ref.build_FockMat()
    K64 = ref.mat("K_mat")
    ref.free()
    e = engine(name, tinyscf.K_MIXED)
    e.s.iter = 0
    e.build_FockMat()
    K = e.mat("K_mat")
    e.free()
    err = np.abs(K - K64).max()
    # ~16 bits per operand, FP32 accumulation
    assert err < 2e-5 * max(1.0, np.abs(K64).max()), err


def test_increment_error_shrinks_with_density_change():
    """Feed the FP64 SCF's densities to a mixed engine one by one."""
    f = engine("c10h22", tinyscf.K_FP64)
    m = engine("c10h22", tinyscf.K_MIXED)
    errs, dDs = [], []
    Dprev = None
    for it in range(10):
        f.s.iter = it
        f.build_FockMat()
        D, C = f.mat("D_mat"), f.mat("Cocc_mat")
        m.set_density(D, C)
        m.s.iter = it
        m.build_FockMat()
        errs.append(np.abs(m.mat("K_mat") - f.mat("K_mat")).max())
        dDs.append(np.inf if Dprev is None else np.abs(D - Dprev).max())
        Dprev = D
        f.DIIS()
        f.build_DenMat()
    f.free()
    m.free()
    # later increments add far less error than the first (full) build carried
    inc = np.abs(np.diff(errs))
    assert inc[-1] < 0.05 * errs[0], (errs, dDs)


@pytest.mark.parametrize("name", ["c10h22", "c20h42"])
def test_mixed_scf_energy_matches_fp64(name):
    # converge both well below the 1e-8 Eh target so the comparison sees the
    # precision of the exchange build, not where each run happened to stop
    e64 = engine(name, tinyscf.K_FP64)
    e64.s.ene_tol = 1e-10
    e64.do_SCF()
    E64 = e64.energy
    e64.free()
    em = engine(name, tinyscf.K_MIXED)
    em.s.ene_tol = 1e-10
    em.do_SCF()
    Em = em.energy
    em.free()
    assert abs(Em - E64) < 1e-8, (Em, E64)


def test_refine_density_matches_full_eigensolves():
    """Occupied-subspace refinement between full eigensolves converges to the
    same SCF energy and density as a full eigensolve every iteration."""
    e0 = engine("c10h22", tinyscf.K_FP64)
    e0.s.ene_tol = 1e-10
    e0.do_SCF()
    E0, D0, it0 = e0.energy, e0.mat("D_mat"), e0.s.iter
    e0.free()
    e1 = engine("c10h22", tinyscf.K_FP64)
    e1.set_density_solver(tinyscf.DENSITY_REFINE)
    e1.s.ene_tol = 1e-10
    c0 = e1.counters()
    e1.do_SCF()
    c1 = e1.counters()
    E1, D1, it1 = e1.energy, e1.mat("D_mat"), e1.s.iter
    e1.free()
    n_eig, n_ref = c1[3] - c0[3], c1[4] - c0[4]
    assert abs(E1 - E0) < 1e-9, (E1, E0)
    assert np.abs(D1 - D0).max() < 1e-6
    assert n_ref > 0 and n_eig < it1, (n_eig, n_ref, it1, it0)


def test_mixed_refine_scf_energy_matches_fp64():
    e64 = engine("c20h42", tinyscf.K_FP64)
    e64.s.ene_tol = 1e-10
    e64.do_SCF()
    E64 = e64.energy
    e64.free()
    em = engine("c20h42", tinyscf.K_MIXED)
    em.set_density_solver(tinyscf.DENSITY_REFINE)
    em.s.ene_tol = 1e-10
    em.do_SCF()
    Em = em.energy
    em.free()
    assert abs(Em - E64) < 1e-8, (Em, E64)
