"""One animation split at the root (temporalsetinversion_b200.split), on the
CPU: the subtree root boxes, the subtree scenes' semantics against the full
octree (oracle), the nearest-depth composite against the full trace, and the
cross-rank exchange of split.combine_ranks with two and three gloo ranks."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
import split_ref
from temporalsetinversion_b200 import api, scenes, split

ROOT = Path(__file__).resolve().parents[1]


def _key(c):
    return np.lexsort((c["iz"], c["iy"], c["ix"], c["level"]))


@pytest.mark.parametrize("level", [1, 2])
def test_subtree_root_boxes_are_the_full_octrees_cells(level):
    """tsi_params_subtree's box of (level, ix, iy, iz) equals that cell's
    bounds in the full octree bit for bit."""
    oracle.build()
    tape = api.IR.new(scenes.spheres16(0)).gpu_instructions
    p = api.default_params(localsubdiv=5, pointsample=0)
    S = oracle.Scene(tape, p)
    S.invert(0.0)
    n = 1 << level
    seen = 0
    for c in S.cells():
        if c["level"] != level:
            continue
        idx = int(c["ix"]) + n * (int(c["iy"]) + n * int(c["iz"]))
        q = split.subtree_params(p, level, idx)
        for a, ax in enumerate("xyz"):
            assert np.float32(q.root_lo[a]) == c[ax][0] and np.float32(q.root_hi[a]) == c[ax][1], (idx, ax)
        assert q.localsubdiv == p.localsubdiv and q.delta == p.delta
        seen += 1
    assert seen >= 8


def test_subtree_params_rejects_bad_arguments():
    p = api.default_params(localsubdiv=4)
    with pytest.raises(Exception):
        split.subtree_params(p, 1, 8)
    with pytest.raises(Exception):
        split.subtree_params(p, 4, 0)  # not below localsubdiv
    assert split.subtree_ids(1, 1, 3) == [1, 4, 7]
    assert sorted(sum((split.subtree_ids(2, r, 5) for r in range(5)), [])) == list(range(64))


@pytest.mark.parametrize("text", [scenes.spheres16(0), scenes.csg(24, 3, 0.9)], ids=["spheres16", "csg24"])
def test_fresh_subtrees_equal_the_full_octree(text):
    """On a fresh octree every subtree scene's cells are the full octree's
    cells of that subtree, all fields bit for bit (subtrees whose root the
    full octree subdivides)."""
    oracle.build()
    tape = api.IR.new(text).gpu_instructions
    p = api.default_params(localsubdiv=6, lipschitz_corrected=1)
    full = oracle.Scene(tape, p)
    full.invert(0.0)
    fc = full.cells()
    compared = 0
    for k in range(8):
        root = fc[(fc["level"] == 1) & (fc["ix"] == k % 2) & (fc["iy"] == (k // 2) % 2) & (fc["iz"] == k // 4)]
        assert len(root) == 1
        if not root[0]["has_children"]:
            continue
        part = oracle.Scene(tape, split.subtree_params(p, 1, k))
        part.invert(0.0)
        pc = split.subtree_cell_keys(part.cells(), 1, k)
        pc = pc[pc["level"] > 1]
        sub = fc[(fc["level"] > 1) & ((fc["ix"] >> (fc["level"] - 1)) == k % 2) &
                 ((fc["iy"] >> (fc["level"] - 1)) == (k // 2) % 2) & ((fc["iz"] >> (fc["level"] - 1)) == k // 4)]
        pc, sub = pc[_key(pc)], sub[_key(sub)]
        assert len(pc) == len(sub) > 8
        assert pc.tobytes() == sub.tobytes(), k
        compared += 1
    assert compared >= 4, compared


def test_composite_matches_the_full_trace():
    """The composite of the eight subtrees' frames shows the full trace's
    picture: the same hit pixels but for a few on silhouettes, depths within
    1e-3 (the rays take other float steps through the parts), normals of the
    same leaves."""
    oracle.build()
    tape = api.IR.new(scenes.csg(24, 3, 0.9)).gpu_instructions
    p = api.default_params(localsubdiv=6, lipschitz_corrected=1)
    u = api.make_uniforms(scenes.camera_look_at((1.2, 0.8, 1.4)), (96, 54), 1.0 / 60.0)
    times = [0.0, 1.0 / 60.0]
    full = oracle.Scene(tape, p)
    for t in times:
        full.invert(t)
    ref = full.trace(u)
    comp = split_ref.composite(split_ref.oracle_parts(tape, p, 1, list(range(8)), times, u), list(range(8)))
    hit_f, hit_c = ref["depth"] >= 0, comp["depth"] >= 0
    assert hit_f.sum() > 500
    assert (hit_f != hit_c).sum() <= 0.01 * hit_f.size
    both = hit_f & hit_c
    assert np.max(np.abs(ref["depth"][both] - comp["depth"][both])) <= 1e-3
    same_n = np.all(ref["normal"][both] == comp["normal"][both], axis=-1)
    assert same_n.mean() > 0.97, same_n.mean()


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_worker(rank: int, world: int, dst: int, port: int, q):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist

    import split_ref as ref
    from temporalsetinversion_b200 import api as A, scenes as SC, split as SP
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    tape = A.IR.new(SC.spheres16(0)).gpu_instructions
    p = A.default_params(localsubdiv=5)
    u = A.make_uniforms(SC.camera_look_at((0.5, 0.5, 1.3)), (48, 27), 0.0)
    ids = SP.subtree_ids(1, rank, world)
    mine = ref.composite(ref.oracle_parts(tape, p, 1, ids, [0.0], u), ids)
    fb = {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in mine.items()}

    def keep(frame, gkey):
        arrs = {k: v.numpy() for k, v in frame.items()}
        ref.keep_nearest(arrs, gkey.numpy())

    out = SP.combine_ranks(fb, keep, dst=dst)
    if rank == dst:
        q.put({k: v.numpy().copy() for k, v in out.items()})
    else:
        q.put(out)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,dst", [(2, 0), (3, 2)])
def test_ranks_combine_to_the_single_rank_composite(world, dst):
    """gloo ranks holding every world-th subtree ({0, 2, 4, 6} and
    {1, 3, 5, 7}; or {0, 3, 6}, {1, 4, 7}, {2, 5}): the MIN all-reduce of
    keys, keep-nearest and SUM reduce of bits give rank `dst` the one-rank
    composite of all eight subtrees bit for bit."""
    import torch.multiprocessing as mp
    oracle.build()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_worker, args=(r, world, dst, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=180) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    merged = [g for g in got if g is not None]
    assert len(merged) == 1
    merged = merged[0]
    tape = api.IR.new(scenes.spheres16(0)).gpu_instructions
    p = api.default_params(localsubdiv=5)
    u = api.make_uniforms(scenes.camera_look_at((0.5, 0.5, 1.3)), (48, 27), 0.0)
    want = split_ref.composite(split_ref.oracle_parts(tape, p, 1, list(range(8)), [0.0], u), list(range(8)))
    assert (want["depth"] >= 0).sum() > 100
    for name in ("rgba", "depth", "normal", "key"):
        assert merged[name].tobytes() == want[name].tobytes(), name
