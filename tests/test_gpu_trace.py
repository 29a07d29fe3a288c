"""Octree ray tracing on the GPU against the oracle's restatement of
compute.wgsl `trace` / `rt_main`: depth, normal and colour images bit for
bit, with stored and finite-difference normals, normal visualisation, the
per-scene cameras, render mode and asynchronous read-back."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from golden.make_golden import load_tape
from temporalsetinversion_b200 import Scene, Tape, api, scenes

def _compare(g, o):
    bad = [k for k in ("depth", "normal", "rgba") if g[k].tobytes() != o[k].tobytes()]
    assert not bad, "images differ: %s" % {k: int((g[k] != o[k]).sum()) for k in bad}


@pytest.mark.gpu
@pytest.mark.parametrize("name,src,params,eye", [
    ("spheres16", "spheres16", dict(localsubdiv=7, pointsample=0), (0.3, 0.6, 2.5)),
    ("csg48", "csg48", dict(localsubdiv=7), (-1.5, 1.0, 2.0)),
    ("sponza", "sponza", dict(localsubdiv=6, normal_viz=1), (0.0, 0.0, 8.0)),
    # normals by finite differences of the tape (compute.wgsl:4143-4184 for any scene)
    ("sponza_fast", "sponza", dict(localsubdiv=6, normal_viz=1, fast_normals=1), (0.0, 0.0, 8.0)),
    ("spheres16_fast", "spheres16", dict(localsubdiv=7, pointsample=0, normal_viz=1, fast_normals=1),
     (0.3, 0.6, 2.5)),
])
def test_trace_matches_oracle(device, name, src, params, eye):
    if src == "spheres16":
        tape = api.IR.new(scenes.spheres16(0)).gpu_instructions
    elif src == "csg48":
        tape = api.IR.new(scenes.csg(48, 4)).gpu_instructions
    else:
        tape = load_tape(src)
    p = api.default_params(**params)
    gs = Scene(device, Tape.upload(device, tape), p)
    os_ = oracle.Scene(tape, p)
    times = [0.0, 1 / 60, 2 / 60]
    for t in times:
        gs.invert(t)
        os_.invert(t)
    u = api.make_uniforms(scenes.camera_look_at(eye), (160, 90), times[-1])
    g = gs.trace(u)
    o = os_.trace(u)
    assert (o["depth"] >= 0).sum() > 100, "camera sees the surface"
    _compare(g, o)


@pytest.mark.gpu
def test_trace_scene_offsets(device):
    """scene ids 0/3/4/5 apply rt_main's eye offsets and rotations."""
    tape = load_tape("cradle")
    for sid in (0, 3, 4, 5):
        p = api.default_params(localsubdiv=5, scene_id=sid)
        gs = Scene(device, Tape.upload(device, tape), p)
        os_ = oracle.Scene(tape, p)
        gs.invert(0.0)
        os_.invert(0.0)
        u = api.make_uniforms(scenes.camera_look_at((0.0, 0.0, 0.5), (0.0, 0.0, -1.0)), (64, 48), 0.0)
        _compare(gs.trace(u), os_.trace(u))


@pytest.mark.gpu
def test_rendermode_black(device):
    tape = api.IR.new(scenes.spheres16(0)).gpu_instructions
    gs = Scene(device, Tape.upload(device, tape), api.default_params(localsubdiv=5))
    gs.invert(0.0)
    u = api.make_uniforms(scenes.camera_look_at((0, 0, 2.5)), (32, 32), 0.0, rendermode=1.0)
    g = gs.trace(u)
    assert np.all(g["rgba"] == 0) and np.all(g["depth"] == -1)


@pytest.mark.gpu
def test_trace_async_matches_trace(device):
    """Frames read back asynchronously (pinned buffers, copies overlapping
    the next inversion) equal the synchronous trace's frames."""
    import torch

    text = scenes.csg(24, 5, 0.8)
    params = api.default_params(localsubdiv=6)
    a = Scene(device, Tape.from_llvm_ir(device, text), params)
    b = Scene(device, Tape.from_llvm_ir(device, text), params)
    cam = scenes.camera_look_at((0.5, 0.9, 2.3))
    res = (160, 96)
    bufs = [torch.empty((res[1], res[0], 4), dtype=torch.float32, pin_memory=True) for _ in range(4)]
    want = []
    for f in range(4):
        t = f / 60.0
        u = api.make_uniforms(cam, res, t)
        a.invert(t)
        a.trace_async(u, bufs[f].numpy())
        b.invert(t)
        want.append(b.trace(u, depth=False, normal=False)["rgba"])
    a.trace_wait()
    for f in range(4):
        assert np.array_equal(bufs[f].numpy(), want[f])


@pytest.mark.gpu
def test_pipelined_frames_match_sequential(device):
    """Inversions and traces queued back to back without waiting (frame i's
    copy to host memory overlapping the inversion of frame i + 1) give the
    frames of the sequential invert-then-trace loop: colour, depth and
    normal."""
    import torch

    text = scenes.csg(64, 5, 0.85)
    params = api.default_params(localsubdiv=7)
    a = Scene(device, Tape.from_llvm_ir(device, text), params)
    b = Scene(device, Tape.from_llvm_ir(device, text), params)
    cam = scenes.camera_look_at((0.5, 0.9, 2.3))
    res = (192, 108)
    n = 8
    pin = lambda c: torch.empty((res[1], res[0], c), dtype=torch.float32, pin_memory=True)
    bufs = [(pin(4), pin(1), pin(3)) for _ in range(n)]
    for f in range(n):
        t = f / 30.0
        a.invert_async(t)
        a.trace_async(api.make_uniforms(cam, res, t), *(x.numpy() for x in bufs[f]))
    a.invert_wait()
    a.trace_wait()
    for f in range(n):
        t = f / 30.0
        b.invert(t)
        want = b.trace(api.make_uniforms(cam, res, t))
        rgba, depth, normal = (x.numpy() for x in bufs[f])
        assert np.array_equal(rgba, want["rgba"]), f
        assert np.array_equal(depth.reshape(want["depth"].shape), want["depth"]), f
        assert np.array_equal(normal.reshape(want["normal"].shape), want["normal"]), f

