"""The aux-partitioned Fock build on the device (TinySCF_set_aux_slice,
TinySCF_set_JK, driven by yatscf-df_b200/auxsplit.py): two handles on one GPU,
each holding half of the DF tensor's aux columns, summed once per iteration,
reach the unpartitioned engine's energy in the same number of iterations
(the reduction only reorders sums: energies within 1e-9 Eh); a sliced handle
refuses TinySCF_do_SCF. The multi-process path (one GPU per rank, NCCL
all-reduce) runs the same loop with torch_allreduce; its reduction logic is
covered on the CPU with gloo ranks (test_auxsplit.py)."""
import pytest

import auxsplit
import tinyscf
from conftest import BAS, DFBAS, xyz

pytestmark = pytest.mark.gpu


def _sliced(name, p0, p1):
    e = tinyscf.TinySCF(BAS, DFBAS, xyz(name), 40)
    e.compute_Hcore_Ovlp_mat()
    e.compute_sq_Schwarz_scrvals()
    e.prepare_sparsity()
    e.get_initial_guess()
    e.set_aux_slice(p0, p1)
    e.build_DF_tensor()
    return e


@pytest.mark.parametrize("name", ["water", "c10h22"])
def test_two_slices_match_the_unpartitioned_engine(name):
    full = tinyscf.TinySCF(BAS, DFBAS, xyz(name), 40)
    full.setup()
    full.do_SCF()
    E_ref, it_ref, naux = full.energy, full.s.iter, full.s.df_nbf
    full.free()
    engines = [_sliced(name, p0, p1) for p0, p1 in auxsplit.aux_slices(naux, 2)]
    E = auxsplit.scf(engines)
    assert abs(E[-1] - E_ref) < 1e-9, (E[-1], E_ref)
    assert len(E) == it_ref
    with pytest.raises(tinyscf.TinySCFError):
        engines[0].do_SCF()
    for e in engines:
        e.free()
