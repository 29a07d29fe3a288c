"""Cinematic path tracing (compute.wgsl `cinematic`, get_color_single
4444-4523, getSampleBiased 4429-4438, frand 2451-2472, sunsky 520-677,
get_color_supersample 4620-4648) on the GPU against the oracle's
restatement: colour, depth and normal images bit for bit.  Bounces, shadow
rays, the sky seen by escaping paths, per-scene sun constants, the primary
miss colour with and without see_background, several samples per pixel and
render mode."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from golden.make_golden import load_tape
from temporalsetinversion_b200 import Scene, Tape, api, scenes


def _same(a: np.ndarray, b: np.ndarray) -> bool:
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def _compare(g, o):
    bad = {k: int((~((g[k] == o[k]) | (np.isnan(g[k]) & np.isnan(o[k])))).sum()) for k in ("depth", "normal", "rgba")
           if not _same(g[k], o[k])}
    assert not bad, "images differ: %s" % bad


CASES = [
    # (name, tape source, params, eye, target, time); the eyes of the scene-id
    # cases are placed so that rt_main's eye offset and rotation for that
    # scene (4670-4679) bring the camera in front of the surface
    ("spheres16", "spheres16", dict(localsubdiv=6, pointsample=0, samples=2), (0.3, 0.6, 2.5), (0, 0, 0), 1 / 60),
    ("csg48_bg", "csg48", dict(localsubdiv=6, samples=2, see_background=1), (-1.5, 1.0, 2.0), (0, 0, 0), 0.25),
    ("sponza_scene3", "sponza", dict(localsubdiv=5, scene_id=3, samples=1, see_background=1), (-7.7, 2.21, -2.7),
     (-7.7, 2.21, -1.7), 0.5),
    ("cradle_scene4", "cradle", dict(localsubdiv=5, scene_id=4, samples=2), (0.0, 0.78, 12.0), (0.0, 0.78, 11.0), 0.1),
    ("piano_scene5", "piano", dict(localsubdiv=5, scene_id=5, samples=1, see_background=1), (-7.13, -2.14, 10.6),
     (-8.13, -2.14, 10.6), 0.3),
    ("spheres16_8spp", "spheres16", dict(localsubdiv=6, samples=8, see_background=1), (0.2, 1.2, 2.2), (0, 0, 0), 0.7),
]


def _tape(src):
    if src == "spheres16":
        return api.IR.new(scenes.spheres16(0)).gpu_instructions
    if src == "csg48":
        return api.IR.new(scenes.csg(48, 4)).gpu_instructions
    return load_tape(src)


@pytest.mark.gpu
@pytest.mark.parametrize("name,src,params,eye,target,t", CASES, ids=[c[0] for c in CASES])
def test_cinematic_matches_oracle(device, name, src, params, eye, target, t):
    tape = _tape(src)
    # path tracing needs normals at every hit: finite differences of the tape
    p = api.default_params(cinematic=1, fast_normals=1, **params)
    gs = Scene(device, Tape.upload(device, tape), p)
    os_ = oracle.Scene(tape, p)
    for tt in (t - 1 / 60, t):
        gs.invert(tt)
        os_.invert(tt)
    u = api.make_uniforms(scenes.camera_look_at(eye, target), (64, 40), t)
    g = gs.trace(u)
    o = os_.trace(u)
    assert (o["depth"] >= 0).sum() > 50, "camera sees the surface"
    lit = o["rgba"][..., :3][o["depth"] >= 0]
    assert np.unique(lit.round(4), axis=0).shape[0] > 10, "shading varies over the surface"
    _compare(g, o)


@pytest.mark.gpu
def test_cinematic_render_mode_is_black(device):
    tape = _tape("spheres16")
    p = api.default_params(cinematic=1, fast_normals=1, localsubdiv=5, samples=2)
    gs = Scene(device, Tape.upload(device, tape), p)
    gs.invert(0.0)
    u = api.make_uniforms(scenes.camera_look_at((0.3, 0.6, 2.5)), (32, 16), 0.0, rendermode=1.0)
    g = gs.trace(u)
    assert np.all(g["rgba"] == 0.0) and np.all(g["depth"] == -1.0)
