"""Multi-process plumbing of bench.py on CPU (gloo, world size 2).

bench.py runs one replica per GPU (each rank its own animation, seed = base
seed + rank) and combines ranks only on the host: the timed region's device
time is the maximum over ranks, frames are summed.  This test runs that
plumbing with two CPU processes."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank: int, world: int, port: int, out):
    sys.path.insert(0, str(ROOT))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    r, w, local = bench.dist_env()
    dist = bench.init_dist(w)
    text, params, view = bench.build_workload(bench.WORKLOAD["seed"] + r)
    bench.barrier(dist)
    mx = bench.reduce_max(dist, 10.0 + r)
    sm = bench.reduce_sum(dist, 3.0)
    out.put((r, local, mx, sm, hash(text), params.localsubdiv))
    dist.destroy_process_group()


def test_two_rank_replica_plumbing():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1] and [r[1] for r in res] == [0, 1]
    assert all(r[2] == 11.0 for r in res)      # max over ranks
    assert all(r[3] == 6.0 for r in res)       # frames summed
    assert res[0][4] != res[1][4]              # each replica renders its own scene
    assert all(r[5] == 10 for r in res)
