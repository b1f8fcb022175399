"""The aux-partitioned SCF driver (yatscf-df_b200/auxsplit.py) on the CPU:
two gloo ranks, each holding half of the DF tensor's aux columns in a stand-in
engine built on the numpy restatement, reduce [J | K] once per iteration and
reproduce the unpartitioned restatement's energies to rounding; the slices
cover the aux index exactly once; partial J and K of the slices sum to the
full ones. No GPU is needed."""
import os
import socket
import types

import numpy as np
import torch.multiprocessing as mp

import auxsplit
import oracle
from conftest import BAS, DFBAS, xyz


class OracleSlice:
    """The handle interface auxsplit.scf drives, on the restatement, holding
    only the aux columns [p0, p1) of the DF tensor."""

    def __init__(self, name, p0, p1):
        o = oracle.OracleSCF(BAS, DFBAS, xyz(name), 40)
        o.setup()
        o.df_tensor = np.ascontiguousarray(o.df_tensor[:, p0:p1])
        o.naux = p1 - p0
        self.o = o
        self.s = types.SimpleNamespace(nbasfuncs=o.nbf, iter=0, HF_energy=0.0, nuc_energy=o.nuc_energy,
                                       ene_tol=oracle.ENE_TOL, niters=40)

    def build_FockMat(self):
        self.o.build_FockMat()

    def mat(self, name):
        return {"J_mat": self.o.J, "K_mat": self.o.K}[name]

    def set_JK(self, J, K):
        o = self.o
        o.J, o.K = J.copy(), K.copy()
        o.F = o.H + 2.0 * o.J - o.K
        o.calc_energy()
        self.s.HF_energy = o.HF_energy

    def DIIS(self):
        self.o.DIIS(self.s.iter)

    def build_DenMat(self):
        self.o.build_DenMat()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, naux, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    p0, p1 = auxsplit.aux_slices(naux, world)[rank]
    out[rank] = auxsplit.scf([OracleSlice("water", p0, p1)], auxsplit.torch_allreduce(dist))
    dist.destroy_process_group()


def test_slices_cover_the_aux_index_once():
    for naux, parts in ((96, 2), (3870, 8), (7, 3), (5, 5)):
        sl = auxsplit.aux_slices(naux, parts)
        assert sl[0][0] == 0 and sl[-1][1] == naux
        assert all(a[1] == b[0] for a, b in zip(sl, sl[1:]))
        assert max(p1 - p0 for p0, p1 in sl) - min(p1 - p0 for p0, p1 in sl) <= 1


def test_partial_jk_sum_to_the_full_build():
    full = oracle.OracleSCF(BAS, DFBAS, xyz("water"), 40)
    full.setup()
    full.build_FockMat()
    J, K = np.zeros_like(full.J), np.zeros_like(full.K)
    for p0, p1 in auxsplit.aux_slices(full.naux, 3):
        part = OracleSlice("water", p0, p1)
        part.build_FockMat()
        J += part.o.J
        K += part.o.K
    assert np.abs(J - full.J).max() < 1e-12 and np.abs(K - full.K).max() < 1e-12


def test_two_gloo_ranks_reproduce_the_unpartitioned_scf():
    ref = oracle.OracleSCF(BAS, DFBAS, xyz("water"), 40)
    ref.setup()
    E = ref.do_SCF()
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(world, _free_port(), ref.naux, out), nprocs=world, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1]                       # every rank holds the same replicated state
    assert len(res[0]) == len(E)
    assert np.abs(np.array(res[0]) - np.array(E)).max() < 1e-10
