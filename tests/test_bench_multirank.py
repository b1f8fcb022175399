"""The N > 1 plumbing of bench.py on the CPU: two gloo ranks agree on the
slowest rank's time (the whole-job device time), and the waters256 work split
covers every cluster exactly once. No GPU is needed."""
import importlib.util
import os
import socket

import torch.multiprocessing as mp

from conftest import REPO


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(REPO, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    b = _bench()
    out[rank] = b.reduce_max(10.0 + 5.0 * rank, dist)
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_to_the_slowest():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        assert dict(out) == {0: 15.0, 1: 15.0}


def test_shards_cover_every_cluster_once():
    b = _bench()
    for world in (1, 2, 3, 8):
        parts = [b.shard(range(256), r, world) for r in range(world)]
        flat = sorted(x for p in parts for x in p)
        assert flat == list(range(256))
        assert max(map(len, parts)) - min(map(len, parts)) <= 1
    assert b.reduce_max(3.5, None) == 3.5
