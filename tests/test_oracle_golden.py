"""Pins the numpy restatement (oracle/oracle.py) against outputs of the
reference's own SCF code (oracle/_ref/ref_dump, compiled from the reference
sources) stored in tests/golden/*_ref.npz."""
import os

import numpy as np
import pytest

import oracle
from conftest import BAS, DFBAS, GOLDEN, xyz


@pytest.fixture(scope="module")
def water():
    g = np.load(os.path.join(GOLDEN, "water_ref.npz"))
    o = oracle.OracleSCF(BAS, DFBAS, xyz("water"), 30)
    o.setup()
    return o, g


def test_water_setup_matches_reference(water):
    o, g = water
    assert np.abs(o.S - g["S"]).max() < 1e-14
    assert np.abs(o.H - g["H"]).max() < 1e-12
    assert np.abs(o.X - g["X"]).max() < 1e-11
    assert (o.bf_pair_mask == g["mask"]).all()
    assert np.abs(o.D - g["D0"]).max() == 0.0
    assert np.abs(o.Cocc - g["Cocc0"]).max() < 1e-14
    assert np.abs(o.df_tensor - g["B"]).max() < 1e-9
    assert abs(o.nuc_energy - float(g["nuc_energy"])) < 1e-12


def test_water_scf_matches_reference(water):
    o, g = water
    seen = {}

    def cb(it, s):
        if it <= 2:
            seen[it] = (s.J.copy(), s.K.copy(), s.F.copy())

    E = np.array(o.do_SCF(cb))
    assert len(E) == len(g["energies"])
    assert np.abs(E - g["energies"]).max() < 1e-10
    for it in (0, 1, 2):
        J, K, F = seen[it]
        assert np.abs(J - g["it%d_J" % it]).max() < 1e-10
        assert np.abs(K - g["it%d_K" % it]).max() < 1e-10
        assert np.abs(F - g["it%d_F" % it]).max() < 1e-10


def test_c10h22_matches_reference():
    g = np.load(os.path.join(GOLDEN, "c10h22_ref.npz"))
    o = oracle.OracleSCF(BAS, DFBAS, xyz("c10h22"), 30)
    o.setup()
    assert (o.bf_pair_mask == g["mask"]).all()
    assert np.abs(o.Cocc - g["Cocc0"]).max() < 1e-12
    J = o.build_J(o.D)
    K = o.build_K(o.Cocc)
    assert np.abs(J - g["it0_J"]).max() < 1e-8
    assert np.abs(K - g["it0_K"]).max() < 1e-8
    E = np.array(o.do_SCF())
    # |dE| < 1e-11 stops the loop at the rounding floor of this ill-conditioned
    # metric (Jpq^-1/2 differs at 1e-3 between LAPACK builds), so iteration
    # counts may differ; the converged energy and the common trajectory may not.
    n = min(len(E), len(g["energies"]))
    assert n >= 10
    assert abs(E[-1] - g["energies"][-1]) < 1e-8
    assert np.abs(E[:n] - g["energies"][:n]).max() < 1e-8


def test_quicksort_eigval_quirk():
    # build_density.c:22-24: an equal-key swap duplicates an index
    ev = [1.0, 2.0, 2.0, 3.0]
    idx = [0, 1, 2, 3]
    oracle.OracleSCF.quickSort_eigval(ev, idx, 0, 3)
    assert ev == sorted(ev)
    assert idx != [0, 1, 2, 3]
