"""The exchange's rank-k product K = T T^T (build_Fock.c:317-341) on the
integer tensor cores (Ozaki scheme II: int8 residues modulo 15 coprime
moduli, exact int32 sums, Chinese-remainder reconstruction), through the C ABI.

* Integer-valued T: every step is exact, so K must equal the exact product bit
  for bit.
* Random T (zero rows, rows scaled by up to 1e+-80, sizes off every tile and
  K-range boundary, odd row pitches): within 2^-47 of each row's scale against an
  80-bit-accumulated product (the only rounding before the last is that of
  each row to a 49-bit integer, 2^-50 of its largest element).
* In the engine (TINYSCF_OZAKI=1 against =0, which runs the FP64 DMMA/FFMA
  kernels): K of the first Fock build within 1e-12 of max|K|, and the same
  converged energy to 1e-10 Eh, on C10H22 and C20H42."""
import os

import numpy as np
import pytest

import tinyscf
from conftest import DATA

pytestmark = pytest.mark.gpu


def _exact(T):
    Tl = T.astype(np.longdouble)
    return (Tl @ Tl.T)


@pytest.mark.parametrize("n,q", [(1, 1), (3, 5), (24, 300), (129, 1000), (257, 4097), (40, 131073)])
def test_integer_valued_is_exact(n, q):
    rng = np.random.default_rng(n * 1000 + q)
    T = rng.integers(-4096, 4097, size=(n, q)).astype(np.float64)
    K = tinyscf.syrk_int8(T)
    ref = (T.astype(np.int64) @ T.astype(np.int64).T).astype(np.float64)   # |sums| < 2^53: exact
    assert np.array_equal(K, ref)


@pytest.mark.parametrize("n,q", [(7, 129), (130, 2001), (255, 8191), (300, 9001)])
def test_random_within_row_scale(n, q):
    rng = np.random.default_rng(n + q)
    T = rng.standard_normal((n, q))
    T[rng.random((n, q)) < 0.3] = 0.0
    T[n // 2] = 0.0                                             # a zero row
    scales = 10.0 ** rng.uniform(-80, 80, size=n)
    scales[:3] = 1.0
    T *= scales[:, None]
    K = tinyscf.syrk_int8(T)
    ref = _exact(T)
    assert np.all(K[n // 2] == 0.0) and np.all(K[:, n // 2] == 0.0)
    assert np.array_equal(K, K.T)
    rmax = np.abs(T).max(axis=1)
    l1 = np.abs(T).sum(axis=1)
    bound = 2.0 ** -47 * (rmax[:, None] * l1[None, :] + l1[:, None] * rmax[None, :]) + 1e-300
    err = np.abs(K.astype(np.longdouble) - ref).astype(np.float64)
    assert np.all(err <= bound), float((err / bound).max())


def test_same_as_fp64_on_a_dense_product():
    rng = np.random.default_rng(5)
    T = rng.standard_normal((256, 12000))
    K = tinyscf.syrk_int8(T)
    ref = _exact(T).astype(np.float64)
    assert np.abs(K - ref).max() / np.abs(ref).max() < 1e-15


def _first_fock_K_and_energy(mol, mode, monkeypatch):
    monkeypatch.setenv("TINYSCF_OZAKI", mode)
    e = tinyscf.TinySCF(os.path.join(DATA, "cc-pvdz", "cc-pvdz.gbs"),
                        os.path.join(DATA, "cc-pVDZ-RI", "cc-pVDZ-RI.gbs"), os.path.join(DATA, mol + ".xyz"), 40)
    try:
        e.setup()
        e.s.iter = 0
        e.build_FockMat()
        K = e.mat("K_mat")
        e.reset_scf()
        e.s.ene_tol = 1e-10
        e.do_SCF()
        return K, e.energy, e.counters()[7]
    finally:
        e.free()


@pytest.mark.parametrize("mol", ["c10h22", "c20h42"])
def test_engine_exchange_matches_fp64_kernels(mol, monkeypatch):
    K0, E0, n0 = _first_fock_K_and_energy(mol, "0", monkeypatch)
    K1, E1, n1 = _first_fock_K_and_energy(mol, "1", monkeypatch)
    assert n0 == 0 and n1 >= 2
    assert np.abs(K1 - K0).max() <= 1e-12 * np.abs(K0).max()
    assert abs(E1 - E0) < 1e-10, (E0, E1)


@pytest.mark.parametrize("mol", ["c10h22", "c20h42"])
def test_half_transform_variants_agree(mol, monkeypatch):
    """The FP64 half-transform's tile variants (the autotuner's candidates for
    build_Fock.c:259-285) give the same K: the 64 x 256 pipelined DMMA tiles
    (3) against the 168 x 128 ones (4), both with the integer-tensor-core
    rank-k product that takes its row scales from them."""
    Ks = {}
    for variant in ("3", "4"):
        monkeypatch.setenv("TINYSCF_KHALF", variant)
        monkeypatch.setenv("TINYSCF_OZAKI", "1")
        e = tinyscf.TinySCF(os.path.join(DATA, "cc-pvdz", "cc-pvdz.gbs"),
                            os.path.join(DATA, "cc-pVDZ-RI", "cc-pVDZ-RI.gbs"), os.path.join(DATA, mol + ".xyz"), 10)
        try:
            e.setup()
            e.s.iter = 0
            e.build_FockMat()
            Ks[variant] = e.mat("K_mat").copy()
        finally:
            e.free()
    assert np.abs(Ks["4"] - Ks["3"]).max() <= 1e-13 * np.abs(Ks["3"]).max()
