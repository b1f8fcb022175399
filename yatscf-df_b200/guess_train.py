"""Train the learned initial guess from densities this engine converges.

Training molecules (all seeded, nothing read from outside the repository):
  * water clusters from geometry.water_cluster(seed), seeds 10000, 10001, ...;
  * alkanes C_nH_(2n+2), n = 2..10, from geometry.alkane(n) with every atom
    displaced by N(0, 0.03 A) per coordinate and a random rigid rotation,
    seeds 20000, 20001, ...
Each is converged by the engine (FP64 K, projected-SAD guess, 1e-8 Eh); its density
gives one training row per atom pair (TinySCF_guess_dataset). The five block
networks are then trained on the GPU by the engine's own kernels
(TinySCF_guess_train) and written to the weights file.

Two ways to converge the training molecules:
  * one by one, in --workers processes that share the GPU;
  * --batched: in waves through the batched SCF (TinySCF_batch_do_SCF: one
    launch per SCF phase over the whole wave), the autotuner off, so that set-up
    is the engines' own work and no timing runs are made for each new size.
    A wave grows until less than --reserve-gb of device memory is free.

    python guess_train.py --waters 512 --alkanes 96 --out guess_weights.bin
    python guess_train.py --batched --waters 4096 --alkanes 256 --epochs 300 ...
"""
import argparse
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import geometry  # noqa: E402
import tinyscf  # noqa: E402


def jittered_alkane(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 11))
    atoms = geometry.alkane(n)
    xyz = np.array([a[1:] for a in atoms])
    xyz = xyz + rng.normal(scale=0.03, size=xyz.shape)
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    xyz = xyz @ geometry._rotation(q).T
    return [(a[0], float(r[0]), float(r[1]), float(r[2])) for a, r in zip(atoms, xyz)]


def training_jobs(waters, alkanes):
    """(tag, atoms) of the training molecules: water clusters of seeds 10000, ...,
    10000 + waters - 1, then jittered alkanes of seeds 20000, ..., 20000 + alkanes - 1."""
    jobs = [("w%d" % s, geometry.water_cluster(s)) for s in range(10000, 10000 + waters)]
    jobs += [("a%d" % s, jittered_alkane(s)) for s in range(20000, 20000 + alkanes)]
    return jobs


def converge(atoms, bas, dfbas, tmpdir, tag, ene_tol=1e-8, guess=None, weights=None, kmode=None, fast=False):
    """Run one SCF; returns (results dict, (features, targets, types) of its converged density).
    fast: projected-SAD guess, subspace-refinement density solver and CUDA-graph
    iterations (FP64 K throughout), which converge to the same density sooner."""
    path = os.path.join(tmpdir, tag + ".xyz")
    geometry.write_xyz(path, atoms)
    e = tinyscf.TinySCF(bas, dfbas, path, 100)
    try:
        t0 = time.perf_counter()
        e.setup()
        if guess is not None:
            e.set_guess(guess, weights)
            e.reset_scf()
        if fast:
            e.set_guess(tinyscf.GUESS_SAD_PROJECTED)
            e.reset_scf()
            e.set_density_solver(tinyscf.DENSITY_REFINE)
            e.set_graph(True)
        if kmode is not None:
            e.set_k_precision(kmode)
        e.s.ene_tol = ene_tol
        e.do_SCF()
        out = dict(energy=e.energy, iters=e.s.iter, nbf=e.s.nbasfuncs, scf_ms=e.timings()["SCF"],
                   wall_s=time.perf_counter() - t0, guess_used=e.guess_used())
        D = e.mat("D_mat")
        data = e.guess_dataset(D)
    finally:
        e.free()
    return out, data


def _worker(args):
    """Converge one shard of molecules in a fresh process (own CUDA context)."""
    jobs, bas, dfbas = args
    tinyscf.load_library()
    feats, tgts, types, iters = [], [], [], []
    with tempfile.TemporaryDirectory() as td:
        for tag, atoms in jobs:
            res, (f, t, y) = converge(atoms, bas, dfbas, td, tag, fast=True)
            feats.append(f)
            tgts.append(t)
            types.append(y)
            iters.append(res["iters"])
    return feats, tgts, types, iters


def generate(jobs, bas, dfbas, workers):
    """Training rows for all jobs; shards run as separate processes on the same GPU."""
    import multiprocessing as mp
    shards = [(jobs[k::workers], bas, dfbas) for k in range(workers)]
    if workers == 1:
        outs = [_worker(shards[0])]
    else:
        with mp.get_context("spawn").Pool(workers) as pool:
            outs = pool.map(_worker, shards)
    feats, tgts, types, iters = [], [], [], []
    for f, t, y, it in outs:
        feats += f
        tgts += t
        types += y
        iters += it
    return feats, tgts, types, iters


def generate_batched(jobs, bas, dfbas, reserve_gb, guess=tinyscf.GUESS_SAD_PROJECTED, ene_tol=1e-8, max_iter=100):
    """Training rows for all jobs from the batched SCF (FP64 K, full eigensolves),
    largest molecules first so that a wave holds molecules of similar size.
    Returns (features, targets, types, iterations, waves, unconverged tags);
    a molecule that used all max_iter iterations gives no rows."""
    tinyscf.load_library()
    tinyscf.set_autotune(False)
    order = sorted(range(len(jobs)), key=lambda k: -len(jobs[k][1]))
    feats, tgts, types, iters, unconverged = [], [], [], [], []
    waves = 0
    with tempfile.TemporaryDirectory() as td:
        k = 0
        while k < len(order):
            wave = []
            try:
                while k < len(order):
                    tag, atoms = jobs[order[k]]
                    k += 1
                    path = os.path.join(td, tag + ".xyz")
                    geometry.write_xyz(path, atoms)
                    e = tinyscf.TinySCF(bas, dfbas, path, max_iter)
                    wave.append((tag, e))
                    e.setup(guess=guess)
                    e.s.ene_tol = ene_tol
                    if tinyscf.device_memory()[0] < reserve_gb * 2 ** 30:
                        break
                b = tinyscf.TinySCFBatch([e for _, e in wave])
                try:
                    b.do_SCF()
                finally:
                    b.free()
                waves += 1
                for tag, e in wave:
                    if e.s.iter >= max_iter:
                        unconverged.append(tag)
                        continue
                    f, t, y = e.guess_dataset(e.mat("D_mat"))
                    feats.append(f)
                    tgts.append(t)
                    types.append(y)
                    iters.append(e.s.iter)
            finally:
                for _, e in wave:
                    e.free()
    return feats, tgts, types, iters, waves, unconverged


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--waters", type=int, default=512)
    ap.add_argument("--alkanes", type=int, default=96)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=os.path.join(HERE, "guess_weights.bin"))
    ap.add_argument("--report", default=None, help="JSON summary path")
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--batched", action="store_true", help="converge the molecules in waves of the batched SCF")
    ap.add_argument("--reserve-gb", type=float, default=40.0,
                    help="--batched: close a wave when less than this much device memory is free")
    ap.add_argument("--bas", required=True)
    ap.add_argument("--dfbas", required=True)
    args = ap.parse_args()

    t0 = time.perf_counter()
    jobs = training_jobs(args.waters, args.alkanes)
    extra = {}
    if args.batched:
        feats, tgts, types, iters, waves, unconverged = generate_batched(jobs, args.bas, args.dfbas, args.reserve_gb)
        extra = dict(mode="batched", waves=waves, unconverged=unconverged, autotune="off")
    else:
        feats, tgts, types, iters = generate(jobs, args.bas, args.dfbas, args.workers)
        extra = dict(mode="one by one", workers=args.workers)
    stats = dict(molecules=len(jobs), pairs=sum(len(y) for y in types), iters=iters)
    gen_s = time.perf_counter() - t0
    F = np.concatenate(feats)
    T = np.concatenate(tgts)
    Y = np.concatenate(types)
    tinyscf.load_library()
    t1 = time.perf_counter()
    loss = tinyscf.guess_train(F, T, Y, args.out, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=0)
    train_s = time.perf_counter() - t1
    rep = dict(molecules=stats["molecules"], pairs=int(stats["pairs"]),
               pairs_per_type=[int((Y == k).sum()) for k in range(5)],
               mean_iterations=float(np.mean(stats["iters"])), data_generation_s=gen_s, training_s=train_s,
               final_loss_per_type=[float(v) for v in loss], weights=os.path.basename(args.out),
               epochs=args.epochs, batch=args.batch, lr=args.lr, **extra)
    print(json.dumps(rep))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
