"""The serving layer: requests for several scenes, submitted faster than
they run, are fused into batches of distinct scenes, each scene's frames run
in submission order, and the octrees equal those of the plain path."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_cells_equal
from temporalsetinversion_b200 import Device, Scene, Server, Tape, api, scenes


@pytest.mark.gpu
def test_server_matches_plain_path():
    texts = [scenes.csg(24, s, 0.9) for s in (3, 4, 5)] + [scenes.spheres16(1)]
    times = [0.0, 1 / 60, 2 / 60, 3 / 60]
    p = api.default_params(localsubdiv=6)
    with Device() as dev:
        plain = [Scene(dev, Tape.from_llvm_ir(dev, t), p) for t in texts]
        for t in times:
            for s in plain:
                s.invert(t)
        want = [s.cells() for s in plain]
        served = [Scene(dev, Tape.from_llvm_ir(dev, t), p) for t in texts]
        with Server(dev) as srv:
            tickets = [srv.submit(s, t) for t in times for s in served]  # all queued up front
            for tk in tickets:
                stats, lat, _ = srv.poll(tk)
                assert lat > 0.0
            st = srv.stats()
        assert st["completed"] == len(tickets)
        assert st["mean_batch"] > 1.0  # distinct scenes were fused
        assert st["batches"] >= len(times)  # one frame per scene per batch
        for s, w in zip(served, want):
            assert_cells_equal(s.cells(), w)


@pytest.mark.gpu
def test_server_rejects_foreign_scene_and_unknown_ticket():
    with Device() as a, Device() as b:
        s = Scene(b, Tape.from_llvm_ir(b, scenes.spheres16(0)), api.default_params(localsubdiv=4))
        with Server(a) as srv:
            with pytest.raises(Exception):
                srv.submit(s, 0.0)
            assert a.lib.tsi_server_poll(srv.handle, 12345, 0, None) == 12  # TSI_ERR_NOT_FOUND
