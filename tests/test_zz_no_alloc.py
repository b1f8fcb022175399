"""The allocation-free J entry point (TinySCF_build_J_noalloc), for callers
that cannot call cudaMalloc, against the engine's own J build: same density,
same DF tensor, two calls in a row into caller-owned device buffers.

Collected last on purpose: if it fails, a run that stops at the first failure
has already run every other test."""
import ctypes

import numpy as np
import pytest

import tinyscf
from conftest import BAS, DFBAS, xyz

pytestmark = pytest.mark.gpu


def test_build_J_noalloc_matches_engine():
    lib = tinyscf.load_library()
    f = lib.TinySCF_build_J_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp]
    f.restype = ctypes.c_int

    e = tinyscf.TinySCF(BAS, DFBAS, xyz("c10h22"), 30)
    e.setup()
    e.s.iter = 0
    e.build_FockMat()                          # the existing entry point, on the SAD density
    J_ref = e.mat("J_mat")
    D = e.mat("D_mat")
    B = e.df_tensor()                          # rows in the reference's CSR order
    _, pj, displs = e.csr()
    nbf, naux = e.s.nbasfuncs, e.s.df_nbf
    e.free()
    up_i, up_j, up_u = [], [], []
    for i in range(nbf):
        for r in range(displs[i], displs[i + 1]):
            if pj[r] >= i:
                up_i.append(i)
                up_j.append(int(pj[r]))
                up_u.append(r)

    import torch                               # device buffers owned by the caller
    dev = torch.device("cuda", 0)
    dB = torch.from_numpy(B).to(dev)
    dD = torch.from_numpy(D).to(dev)
    di = torch.tensor(up_i, dtype=torch.int32, device=dev)
    dj = torch.tensor(up_j, dtype=torch.int32, device=dev)
    du = torch.tensor(up_u, dtype=torch.int32, device=dev)
    dJ = torch.full((nbf, nbf), float("nan"), dtype=torch.float64, device=dev)
    for _ in range(2):
        rc = f(dB.data_ptr(), naux, di.data_ptr(), dj.data_ptr(), du.data_ptr(), len(up_i), nbf,
               dD.data_ptr(), dJ.data_ptr(), None)
        torch.cuda.synchronize()
        assert rc == 0
        J = dJ.cpu().numpy()
        assert np.abs(J - J_ref).max() < 1e-10
        dJ.fill_(float("nan"))
    # sizes beyond the fixed scratch are refused before any launch
    assert f(dB.data_ptr(), 5000, di.data_ptr(), dj.data_ptr(), du.data_ptr(), len(up_i), nbf,
             dD.data_ptr(), dJ.data_ptr(), None) == 4
