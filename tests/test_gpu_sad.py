"""SAD initial guess (TinySCF.c:282-364): the pivoted Cholesky of the
block-diagonal SAD density (LAPACKE_dpstrf at TinySCF.c:295) skips the other
atoms' exact zeros; its Cocc must equal the dense kernel's bit for bit (same
pivots, same sums: every skipped term is an exact zero)."""
import os

import numpy as np
import pytest

import tinyscf
from conftest import DATA

pytestmark = pytest.mark.gpu


def _sad(mol, blocks, monkeypatch):
    monkeypatch.setenv("TINYSCF_PSTF_BLOCKS", "1" if blocks else "0")
    e = tinyscf.TinySCF(os.path.join(DATA, "cc-pvdz", "cc-pvdz.gbs"),
                        os.path.join(DATA, "cc-pVDZ-RI", "cc-pVDZ-RI.gbs"), os.path.join(DATA, mol + ".xyz"), 10)
    try:
        e.compute_Hcore_Ovlp_mat()
        e.compute_sq_Schwarz_scrvals()
        e.prepare_sparsity()
        e.get_initial_guess()
        return e.mat("Cocc_mat").copy(), e.mat("D_mat").copy(), e.timings()["GUESS"]
    finally:
        e.free()


@pytest.mark.parametrize("mol", ["water", "c10h22", "c40h82"])
def test_block_skipping_cholesky_is_bit_identical(mol, monkeypatch):
    C0, D0, t0 = _sad(mol, False, monkeypatch)
    C1, D1, t1 = _sad(mol, True, monkeypatch)
    assert np.array_equal(C0, C1)
    assert np.array_equal(D0, D1)
