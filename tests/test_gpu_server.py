"""The serving layer.  Continuous batching: requests for several scenes,
submitted all at once or while others run on the device, join the running
inversion at launch-step boundaries; each request's octree, depth and colour
images and counters equal the same request run alone on the plain path (one
tsi_scene_invert + tsi_scene_trace), and a scene's frames run in submission
order.  The static-batch form gives the same results.  The queue is bounded
and a request's frame is admitted against the memory budget at submission."""
from __future__ import annotations

import math
import time

import numpy as np
import pytest

from conftest import assert_cells_equal
from temporalsetinversion_b200 import Device, Scene, Server, Tape, api, scenes
from temporalsetinversion_b200 import _native as N

COUNTERS = ("cells_evaluated", "cells_reverse", "cells_ambiguous", "cells_empty", "cells_full", "cells_enqueued",
            "cells_reused", "cells_skipped", "bricks_allocated", "bricks_freed", "voxels_live")


def _texts():
    # different tapes and depths: a long CSG tape (wide path at the top), short
    # ones, a swept scene
    return [(scenes.csg(96, 3, 0.9), 7, 0), (scenes.csg(24, 4, 0.9), 6, 0), (scenes.spheres16(1), 8, 0),
            (scenes.swept(6, 5), 6, 1)]


def _scene_set(dev):
    out = []
    for text, L, swept in _texts():
        p = api.default_params(localsubdiv=L, swept_volume=swept, lipschitz_corrected=1)
        out.append(Scene(dev, Tape.from_llvm_ir(dev, text), p))
    return out


def _requests(n_per_scene: int, res=(80, 48)):
    """Per scene k, frame f: (k, t, t0, uniforms); a camera per request."""
    rng = np.random.default_rng(7)
    reqs = []
    for f in range(n_per_scene):
        for k, (_, _, swept) in enumerate(_texts()):
            t = 0.1 * k + f / 60.0 if f != 2 else 0.77  # one jump in time
            t0 = t - 1.0 / 60.0 if swept else math.nan
            reqs.append((k, t, t0, api.make_uniforms(scenes.camera_on_sphere(rng, 2.5), res, t)))
    return reqs


def _plain(dev, reqs):
    sc = _scene_set(dev)
    out = []
    for k, t, t0, u in reqs:
        st = sc[k].invert(t, t0)
        img = sc[k].trace(u, normal=False)
        out.append((st, img["rgba"], img["depth"]))
    return out, [s.cells() for s in sc]


def _check(results, want, cells_got, cells_want):
    for i, ((st, rgba, depth), (wst, wrgba, wdepth)) in enumerate(zip(results, want)):
        assert st.error_flags == 0
        for c in COUNTERS:
            assert getattr(st, c) == getattr(wst, c), "request %d: %s %d != %d" % (
                i, c, getattr(st, c), getattr(wst, c))
        assert np.array_equal(depth, wdepth), "request %d: depth differs" % i
        assert np.array_equal(rgba, wrgba), "request %d: rgba differs" % i
    for g, w in zip(cells_got, cells_want):
        assert_cells_equal(g, w)


@pytest.mark.gpu
@pytest.mark.parametrize("static", [False, True])
def test_server_requests_equal_plain_path_all_queued(static):
    reqs = _requests(4)
    with Device() as dev:
        want, cells_want = _plain(dev, reqs)
        served = _scene_set(dev)
        with Server(dev, static_batches=static) as srv:
            tickets = [srv.submit(served[k], t, t0=t0, uniforms=u, image=True) for k, t, t0, u in reqs]
            results = []
            for tk in tickets:
                st, lat, rgba, depth = srv.poll(tk, with_depth=True)
                assert lat > 0.0
                results.append((st, rgba, depth))
            ss = srv.stats()
        assert ss["completed"] == len(reqs)
        assert ss["mean_batch"] > 1.0  # requests of distinct scenes ran together
        _check(results, want, [s.cells() for s in served], cells_want)


@pytest.mark.gpu
def test_server_admits_requests_while_others_run():
    """Requests submitted one by one with gaps shorter than a frame: each
    joins the running inversion at a step boundary, and every result is the
    request's own."""
    reqs = _requests(5)
    with Device() as dev:
        want, cells_want = _plain(dev, reqs)
        served = _scene_set(dev)
        with Server(dev) as srv:
            tickets = []
            for k, t, t0, u in reqs:
                tickets.append(srv.submit(served[k], t, t0=t0, uniforms=u, image=True))
                time.sleep(0.0002)
            results = []
            for tk in tickets:
                st, _, rgba, depth = srv.poll(tk, with_depth=True)
                results.append((st, rgba, depth))
            ss = srv.stats()
        assert ss["completed"] == len(reqs) and ss["queued"] == 0
        _check(results, want, [s.cells() for s in served], cells_want)


@pytest.mark.gpu
def test_server_queue_is_bounded():
    with Device() as dev:
        s = Scene(dev, Tape.from_llvm_ir(dev, scenes.csg(64, 2, 0.9)), api.default_params(localsubdiv=8))
        busy = 0
        tickets = []
        with Server(dev, max_queue=2) as srv:
            for i in range(40):  # one scene: its requests run one after another
                try:
                    tickets.append(srv.submit(s, i / 60.0))
                except N.TsiError as e:
                    assert e.status == 11  # TSI_ERR_BUSY: the queue is full
                    busy += 1
                    time.sleep(0.0005)
            for tk in tickets:
                assert srv.poll(tk) is not None
            assert srv.stats()["queued"] == 0
            srv.poll(srv.submit(s, 1.0))  # an empty queue takes requests again
        assert busy > 0 and len(tickets) >= 2


@pytest.mark.gpu
def test_server_admits_frames_against_the_memory_budget():
    with Device() as probe:
        s0 = Scene(probe, Tape.from_llvm_ir(probe, scenes.spheres16(0)), api.default_params(localsubdiv=5))
        scene_bytes = s0.device_bytes()
    budget = scene_bytes + 64 * 64 * 32 + 1024  # the scene plus a 64x64 frame
    with Device(hbm_budget_bytes=budget) as dev:
        s = Scene(dev, Tape.from_llvm_ir(dev, scenes.spheres16(0)), api.default_params(localsubdiv=5))
        cam = scenes.camera_look_at((0.3, 0.6, 2.5))
        with Server(dev) as srv:
            ok = srv.submit(s, 0.0, uniforms=api.make_uniforms(cam, (64, 64), 0.0))
            with pytest.raises(N.TsiError) as e:
                srv.submit(s, 1 / 60, uniforms=api.make_uniforms(cam, (512, 512), 1 / 60))
            assert e.value.status == 4  # TSI_ERR_OOM at submission
            assert srv.poll(ok) is not None


@pytest.mark.gpu
def test_server_rejects_foreign_scene_and_unknown_ticket():
    with Device() as a, Device() as b:
        s = Scene(b, Tape.from_llvm_ir(b, scenes.spheres16(0)), api.default_params(localsubdiv=4))
        with Server(a) as srv:
            with pytest.raises(Exception):
                srv.submit(s, 0.0)
            assert a.lib.tsi_server_poll(srv.handle, 12345, 0, None) == 12  # TSI_ERR_NOT_FOUND
