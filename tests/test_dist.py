"""Rank plumbing of bench.py on CPU: world size 2 over gloo (127.0.0.1).

The layout of one graph is not sharded ("replicas only"): each rank runs its
own replica and the ranks only meet in a barrier and a max-reduction of their
device times, which is what this test exercises.
"""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    r, w, local = bench.dist_env()
    d = bench.Dist(w, local, backend="gloo")
    d.barrier()
    mx = d.max(10.0 * (r + 1))
    d.barrier()
    out[r] = mx
    d.close()


def test_two_rank_barrier_and_max_over_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert dict(out) == {0: 20.0, 1: 20.0}
