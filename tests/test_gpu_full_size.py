"""The configurations the measurements are quoted on, at their full sizes,
against the CPU oracle: the small plain case (16 spheres, localsubdiv 8,
640x360, one frame at t = 0) and the first two frames of the benchmark
animation (256 primitives, localsubdiv 10, 1920x1080).  Octrees cell by
cell, frame counters, and images bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import assert_cells_equal
from temporalsetinversion_b200 import Scene, Tape, api, scenes

COUNTERS = ["parents_expanded", "cells_evaluated", "cells_reverse", "cells_ambiguous", "cells_empty", "cells_full",
            "cells_enqueued", "cells_reused"]


def _run(device, text, params, frames, res, eye, voxels=0):
    tape = api.IR.new(text).gpu_instructions
    gs = Scene(device, Tape.upload(device, tape), params, voxel_capacity=voxels)
    os_ = oracle.Scene(tape, params)
    cam = scenes.camera_look_at(eye)
    for t in frames:
        sg = gs.invert(t).as_dict()
        so = os_.invert(t)
        for k in COUNTERS:
            assert sg[k] == so[k], "t=%g %s: gpu %d oracle %d" % (t, k, sg[k], so[k])
        assert_cells_equal(gs.cells(), os_.cells())
        u = api.make_uniforms(cam, res, t)
        g, o = gs.trace(u), os_.trace(u)
        assert (o["depth"] >= 0).sum() > 1000, "camera sees the surface"
        for key in ("depth", "rgba", "normal"):
            assert np.array_equal(g[key], o[key]), "t=%g: %s differs in %d values" % (
                t, key, int((g[key] != o[key]).sum()))


@pytest.mark.gpu
def test_small_plain_case_spheres16_L8_640x360(device):
    p = api.default_params(localsubdiv=8, delta=0.01, pointsample=0, lipschitz_corrected=0)
    _run(device, scenes.spheres16(0), p, [0.0], (640, 360), (0.3, 0.6, 2.5))


@pytest.mark.gpu
def test_benchmark_animation_first_frames_L10_1080p(device):
    p = api.default_params(localsubdiv=10, delta=0.01, lipschitz_corrected=1, pointsample=1, fast_normals=0)
    _run(device, scenes.csg(256, 1), p, [0.0, 1.0 / 119.0], (1920, 1080), (1.6, 1.0, 1.9), voxels=64 << 20)
