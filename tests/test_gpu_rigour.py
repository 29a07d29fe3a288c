"""Rigour of the directed-rounding mode at the octree level: no cell the
GPU classifies as empty (f = +1) or full (f = -1) may contain a sign change
of f, checked by dense float64 point sampling (tests/point_eval.py) of the
same tape.  Point sampling is off, so every classification rests on an
interval enclosure.  Cells evaluated in the current frame are checked
exactly; a cell carried over from an earlier frame is only guaranteed up to
its ancestors' accumulated time_err (compute.wgsl:3996), checked with that
tolerance (tests/carried_ref.py)."""
from __future__ import annotations

import numpy as np
import pytest

from carried_ref import carried_excursions
from golden.make_golden import load_tape
from point_eval import evaluate
from temporalsetinversion_b200 import Scene, Tape, api, scenes

CASES = {
    "spheres16": (lambda: scenes.spheres16(0), 6),
    "csg24": (lambda: scenes.csg(24, 3, 0.9), 6),
    "csg64": (lambda: scenes.csg(64, 5, 0.85), 6),
}


def _samples(cells: np.ndarray, rng, n_random: int = 24):
    """Corners, centre and random interior points of every cell box."""
    lo = np.stack([cells["x"][:, 0], cells["y"][:, 0], cells["z"][:, 0]], axis=1).astype(np.float64)
    hi = np.stack([cells["x"][:, 1], cells["y"][:, 1], cells["z"][:, 1]], axis=1).astype(np.float64)
    corners = np.array([[(k >> 0) & 1, (k >> 1) & 1, (k >> 2) & 1] for k in range(8)], np.float64)
    u = np.concatenate([corners, [[0.5, 0.5, 0.5]], rng.uniform(size=(n_random, 3))], axis=0)
    return lo[:, None, :] + u[None, :, :] * (hi - lo)[:, None, :]


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_directed_octree_is_rigorous(device, case):
    make, levels = CASES[case]
    text = make()
    tape = api.IR.new(text).gpu_instructions
    p = api.default_params(localsubdiv=levels, pointsample=0, rounding_mode=1)
    s = Scene(device, Tape.upload(device, tape), p)
    rng = np.random.default_rng(11)
    checked = 0
    for t in (0.0, 0.05, 0.1):
        s.invert(t)
        cells = s.cells()
        now = cells[(cells["t"] == np.float32(t)) & (cells["f"] != 0)]
        for sign in (1.0, -1.0):
            sel = now[now["f"] == sign]
            if len(sel) == 0:
                continue
            pts = _samples(sel, rng)
            f = evaluate(tape, pts[..., 0], pts[..., 1], pts[..., 2], np.float64(np.float32(t)))
            bad = np.nonzero(np.any(sign * f <= -1e-9, axis=1))[0]
            assert len(bad) == 0, "%s t=%g: %d cells classified %+d contain f of the other sign, e.g. key %s" % (
                case, t, len(bad), sign, tuple(int(sel[bad[0]][k]) for k in ("level", "ix", "iy", "iz")))
            checked += len(sel)
    assert checked > 100


# the benchmark's 256-primitive tape (4697 slots) and the reference's `cables`
# scene (sin, cos, exp, atan2): a bounded random subset of each frame's
# classified cells is sampled
BIG_CASES = {
    "csg256_L8": (lambda: api.IR.new(scenes.csg(256, 1)).gpu_instructions, 8),
    "cables_L7": (lambda: load_tape("cables"), 7),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(BIG_CASES))
def test_directed_octree_is_rigorous_at_scale(device, case):
    make, levels = BIG_CASES[case]
    tape = make()
    p = api.default_params(localsubdiv=levels, pointsample=0, rounding_mode=1)
    s = Scene(device, Tape.upload(device, tape), p)
    rng = np.random.default_rng(17)
    checked = 0
    for t in (0.0, 0.05, 0.1):
        s.invert(t)
        cells = s.cells()
        now = cells[(cells["t"] == np.float32(t)) & (cells["f"] != 0)]
        for sign in (1.0, -1.0):
            sel = now[now["f"] == sign]
            if len(sel) == 0:
                continue
            sel = sel[rng.choice(len(sel), min(len(sel), 1500), replace=False)]
            pts = _samples(sel, rng, n_random=8)
            f = evaluate(tape, pts[..., 0], pts[..., 1], pts[..., 2], np.float64(np.float32(t)))
            bad = np.nonzero(np.any(sign * f <= -1e-9, axis=1))[0]
            assert len(bad) == 0, "%s t=%g: %d cells classified %+d contain f of the other sign, e.g. key %s" % (
                case, t, len(bad), sign, tuple(int(sel[bad[0]][k]) for k in ("level", "ix", "iy", "iz")))
            checked += len(sel)
    assert checked > 500, checked


@pytest.mark.gpu
@pytest.mark.parametrize("delta", [0.005, 0.02])
def test_directed_swept_volume_has_no_false_empty(device, delta):
    """Swept volume (the union of the shape over each frame's [t0, t]):
    every cell evaluated in the current frame and classified empty is free
    of the surface at float64 samples of space and of its time interval."""
    text = scenes.swept(8, 4)
    tape = api.IR.new(text).gpu_instructions
    p = api.default_params(localsubdiv=6, pointsample=0, rounding_mode=1, swept_volume=1, delta=delta)
    s = Scene(device, Tape.upload(device, tape), p)
    rng = np.random.default_rng(5)
    checked = 0
    for k in range(4):
        t0, t1 = k / 16.0, (k + 1) / 16.0
        s.invert(t1, t0)
        cells = s.cells()
        sel = cells[(cells["t"] == np.float32(t1)) & (cells["f"] == 1.0)]
        if len(sel) == 0:
            continue
        pts = _samples(sel, rng, n_random=12)
        for tt in np.linspace(t0, t1, 5):
            f = evaluate(tape, pts[..., 0], pts[..., 1], pts[..., 2], np.float64(np.float32(tt)))
            bad = np.nonzero(np.any(f <= -1e-9, axis=1))[0]
            assert len(bad) == 0, "t in [%g, %g]: %d empty cells hold f < 0 at t=%g" % (t0, t1, len(bad), tt)
        checked += len(sel)
    assert checked > 50


@pytest.mark.gpu
@pytest.mark.parametrize("lipschitz", [0, 1])
def test_directed_carried_cells_stay_within_ancestors_time_err(device, lipschitz):
    """Directed mode, 40 frames: every empty or full cell carried over from
    an earlier frame keeps its sign at float64 samples up to its ancestors'
    time_err (times |grad f| <= 1 with the Lipschitz correction; the directed
    mode's MIN/MAX hull keeps the correction's gradient bound a lower bound,
    where the reference's (1, 1) rule does not, see
    tests/test_cpu_carried_cells.py).  With the hull every sensitivity
    component of a cell with an undecided min/max contains 0, so lb = 0, df
    becomes delta and the cell is re-enqueued: with the correction few cells
    carry over (4 in these 40 frames), all within the bound."""
    text = scenes.csg(64, 5, 0.85)
    tape = api.IR.new(text).gpu_instructions
    p = api.default_params(localsubdiv=6, pointsample=0, rounding_mode=1, lipschitz_corrected=lipschitz, delta=0.03)
    s = Scene(device, Tape.upload(device, tape), p)
    rng = np.random.default_rng(3)
    checked = 0
    for k in range(40):
        t = k / 60.0
        s.invert(t)
        exc, bound = carried_excursions(tape, s.cells(), t, rng)
        over = exc > bound + 1e-6
        assert not over.any(), "t=%g: %d carried cells cross by more than their ancestors' time_err (%g > %g)" % (
            t, over.sum(), exc[over][0], bound[over][0])
        checked += len(exc)
    assert checked > (50 if lipschitz == 0 else 0), checked
