"""Batched form: many scenes (different tapes, depths, times) in one fused
launch sequence give exactly what each gives alone."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import assert_cells_equal
from temporalsetinversion_b200 import Scene, Tape, api, scenes


def _make(device, specs):
    out = []
    for text, L in specs:
        tape = Tape.from_llvm_ir(device, text)
        out.append(Scene(device, tape, api.default_params(localsubdiv=L)))
    return out


SPECS = [(scenes.csg(16, 1, 0.9), 6), (scenes.spheres16(2), 7), (scenes.csg(40, 3, 0.9), 5), (scenes.swept(6, 5), 6)]


@pytest.mark.gpu
def test_batch_equals_alone(device):
    alone = _make(device, SPECS)
    mixed = _make(device, SPECS)
    times = [[0.0, 0.1, 0.3], [0.2, 0.25, 0.3], [0.9, 0.5, 0.1], [0.0, 1 / 60, 2 / 60]]
    cam = scenes.camera_look_at((0.4, 0.8, 2.4))
    for f in range(3):
        reqs = []
        for i, s in enumerate(mixed):
            u = api.make_uniforms(cam, (96, 64), times[i][f])
            reqs.append((s, times[i][f], math.nan, u))
        res = api.run_batch(device, reqs)
        for i, s in enumerate(alone):
            st = s.invert(times[i][f])
            u = api.make_uniforms(cam, (96, 64), times[i][f])
            img = s.trace(u)
            assert res[i]["stats"].error_flags == 0
            assert_cells_equal(mixed[i].cells(), s.cells())
            assert np.array_equal(res[i]["depth"], img["depth"])
            assert np.array_equal(res[i]["rgba"], img["rgba"])


@pytest.mark.gpu
def test_graph_replays_equal_plain_frames(device):
    """A captured batch replayed over several frames (new times and cameras
    each launch) gives the plain path's octrees and images."""
    alone = _make(device, SPECS[:3])
    graphed = _make(device, SPECS[:3])
    res = (96, 64)
    eyes = [(0.4, 0.8, 2.4), (0.5, 0.7, 2.3), (0.6, 0.6, 2.2)]
    times = [[0.0, 0.2, 0.9], [0.05, 0.25, 0.8], [0.1, 0.3, 0.7]]
    reqs = [(s, times[0][i], math.nan, api.make_uniforms(scenes.camera_look_at(eyes[0]), res, times[0][i]))
            for i, s in enumerate(graphed)]
    g = api.BatchGraph(device, reqs)
    try:
        for f in range(3):
            unis = [api.make_uniforms(scenes.camera_look_at(eyes[f]), res, times[f][i]) for i in range(3)]
            g.launch(times[f], unis)
            st = g.wait()
            assert st.error_flags == 0 and st.device_ms > 0.0 and st.cells_evaluated > 0
            for i, s in enumerate(alone):
                s.invert(times[f][i])
                want = s.trace(unis[i])
                got = graphed[i].image(*res)
                assert_cells_equal(graphed[i].cells(), s.cells())
                assert np.array_equal(got["depth"], want["depth"])
                assert np.array_equal(got["rgba"], want["rgba"])
    finally:
        g.close()
