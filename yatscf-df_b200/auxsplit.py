"""Aux-partitioned SCF of one molecule over several GPUs, one process (and
one engine handle) per GPU.

The DF tensor B(uv, P) enters J and K only through sums over its aux index P:
t(P) = sum_kl D_kl B(kl, P), J = B t, and K = sum_P T_P T_P^T with
T_P(i, s) = sum_j C(j, s) B(ij, P) (build_Fock.c:37-130, 244-347). So the aux
index is cut into contiguous slices, one per rank; each rank builds and holds
only its columns of B (TinySCF_set_aux_slice before TinySCF_build_DF_tensor:
nu x naux/world doubles instead of nu x naux) and its J and K are partial
sums. One all-reduce of [J | K] (2 nbf^2 doubles, 16 MB for C40H82) per
iteration gives every rank the full J and K; the Fock assembly and energy
(TinySCF_set_JK), DIIS and the density are then the same on every rank. The
loop is the reference's, TinySCF.c:378-435.

Several slices can also live in one process (a list of handles, summed
locally before the collective): that is how one GPU runs the partitioned path.
"""
import numpy as np


def aux_slices(naux, parts):
    """Contiguous, balanced slices [p0, p1) covering range(naux)."""
    q, r = divmod(naux, parts)
    out, p0 = [], 0
    for k in range(parts):
        p1 = p0 + q + (1 if k < r else 0)
        out.append((p0, p1))
        p0 = p1
    return out


def torch_allreduce(dist, device=None):
    """Sum of a float64 numpy vector over the ranks of a torch.distributed
    process group (gloo on host tensors, or NCCL with device="cuda:k")."""
    def reduce(x):
        import torch
        t = torch.from_numpy(np.ascontiguousarray(x))
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t)
        return t.cpu().numpy()
    return reduce


def scf(engines, allreduce=None, ene_tol=None, niters=None):
    """The SCF loop over this process's slice handles (all with the same
    molecule and the same initial guess); allreduce sums a vector over the
    processes (None: this process holds every slice). Returns the energy of
    every iteration; the handles end in the state TinySCF_do_SCF leaves."""
    e0 = engines[0]
    tol = e0.s.ene_tol if ene_tol is None else ene_tol
    nit = e0.s.niters if niters is None else niters
    n = e0.s.nbasfuncs
    energies = []
    it, prev, delta = 0, 0.0, 223.0
    while it < nit and delta >= tol:
        jk = np.zeros(2 * n * n)
        for e in engines:
            e.s.iter = it
            e.build_FockMat()                    # this slice's partial J and K
            jk[:n * n] += e.mat("J_mat").ravel()
            jk[n * n:] += e.mat("K_mat").ravel()
        if allreduce is not None:
            jk = allreduce(jk)                   # the one collective of the iteration
        J, K = jk[:n * n].reshape(n, n), jk[n * n:].reshape(n, n)
        for e in engines:
            e.set_JK(J, K)                       # F = H + 2J - K and the energy
        E = e0.s.HF_energy
        delta = abs(E - prev)
        prev = E
        for e in engines:
            e.DIIS()
            e.build_DenMat()
        energies.append(E + e0.s.nuc_energy)
        if it == 0:
            delta = 223.0
        it += 1
    for e in engines:
        e.s.iter = it
    return energies
