"""The wide-path threshold is a speed knob only: every threshold gives the
same octrees and images, and the autotuner keeps one of the thresholds it
timed."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_cells_equal
from temporalsetinversion_b200 import Scene, Tape, api, scenes

NARROW_ONLY = 0xFFFFFFFF


def _frames(device, text, L, threshold, times, res=(96, 64), deep=None, parents=None, prune_level=None):
    tape = Tape.from_llvm_ir(device, text)
    if parents is not None:
        tape.narrow_parents = parents
    if prune_level is not None:
        tape.wide_prune_level = prune_level
    if threshold is not None:
        tape.wide_threshold = threshold
    if deep is not None:
        tape.wide_threshold_deep = deep
    s = Scene(device, tape, api.default_params(localsubdiv=L))
    cam = scenes.camera_look_at((0.5, 0.9, 2.3))
    out = []
    for t in times:
        st = s.invert(t)
        assert st.error_flags == 0
        img = s.trace(api.make_uniforms(cam, res, t))
        out.append((s.cells(), img["depth"], img["rgba"]))
    return tape, out


@pytest.mark.gpu
def test_thresholds_give_identical_frames(device):
    text = scenes.csg(40, 11, 0.8)
    times = [0.0, 1 / 60, 2 / 60, 0.5]
    tape, want = _frames(device, text, 7, NARROW_ONLY, times)
    assert tape.wide_threshold == NARROW_ONLY
    for thr in (16, 128, None):
        _, got = _frames(device, text, 7, thr, times)
        for (wc, wd, wr), (gc, gd, gr) in zip(want, got):
            assert_cells_equal(gc, wc)
            assert np.array_equal(gd, wd)
            assert np.array_equal(gr, wr)


@pytest.mark.gpu
def test_deep_level_thresholds_give_identical_frames(device):
    """A second threshold for the deepest levels (narrow only there, or a
    different length) is a speed knob too."""
    text = scenes.csg(96, 3, 0.9)
    times = [0.0, 1 / 60, 2 / 60]
    _, want = _frames(device, text, 8, None, times)
    for deep in ((6, NARROW_ONLY), (5, 512), (3, 64)):
        tape, got = _frames(device, text, 8, None, times, deep=deep)
        assert tape.wide_threshold_deep == deep
        for (wc, wd, wr), (gc, gd, gr) in zip(want, got):
            assert_cells_equal(gc, wc)
            assert np.array_equal(gd, wd)
            assert np.array_equal(gr, wr)


@pytest.mark.gpu
def test_narrow_parents_give_identical_frames(device):
    """Parents per narrow work item (1, 2 or 4) only change how cells are
    packed onto warps."""
    text = scenes.csg(64, 5, 0.85)
    times = [0.0, 1 / 60, 2 / 60]
    _, want = _frames(device, text, 7, NARROW_ONLY, times, parents=4)
    for parents in (1, 2):
        tape, got = _frames(device, text, 7, NARROW_ONLY, times, parents=parents)
        assert tape.narrow_parents == parents
        for (wc, wd, wr), (gc, gd, gr) in zip(want, got):
            assert_cells_equal(gc, wc)
            assert np.array_equal(gd, wd)
            assert np.array_equal(gr, wr)


@pytest.mark.gpu
def test_wide_prune_levels_give_identical_frames(device):
    """Wide groups above the prune level skip pruning (their children run
    the full tape on the wide path); every prune level gives the same octrees
    and images."""
    text = scenes.csg(96, 7, 0.85)
    times = [0.0, 1 / 60, 2 / 60, 3 / 60]
    _, want = _frames(device, text, 8, 64, times, prune_level=0)
    for level in (2, 4, 0xFFFFFFFF, 99):
        tape, got = _frames(device, text, 8, 64, times, prune_level=level)
        assert tape.wide_prune_level == level
        for (wc, wd, wr), (gc, gd, gr) in zip(want, got):
            assert_cells_equal(gc, wc)
            assert np.array_equal(gd, wd)
            assert np.array_equal(gr, wr)


@pytest.mark.gpu
def test_autotune_keeps_a_timed_threshold(device):
    text = scenes.csg(64, 12, 0.7)
    tape = Tape.from_llvm_ir(device, text)
    s = Scene(device, tape, api.default_params(localsubdiv=7))
    times = [0.1, 0.1 + 1 / 60, 0.1 + 2 / 60]
    r = s.autotune(times, reps=1)
    tried = [thr for thr, _ in r["trials"]]
    assert r["wide_threshold"] in tried and NARROW_ONLY in tried
    assert tape.wide_threshold == r["wide_threshold"]
    assert tape.wide_prune_level == r["wide_prune_level"]
    ms = dict(r["trials"])
    assert ms[r["wide_threshold"]] == min(ms.values())
    # left reset: the next frames match a fresh scene's
    fresh = Scene(device, Tape.from_llvm_ir(device, text), api.default_params(localsubdiv=7))
    for t in times:
        s.invert(t)
        fresh.invert(t)
        assert_cells_equal(s.cells(), fresh.cells())


@pytest.mark.gpu
def test_global_working_set_matches_narrow(device):
    """A tape whose wide working set exceeds shared memory (about 12k
    slots) runs its wide cells from global scratch, with the narrow path's
    results."""
    text = scenes.csg(700, 13, 0.7)
    times = [0.2, 0.2 + 1 / 60, 0.6]
    tape, want = _frames(device, text, 6, NARROW_ONLY, times)
    assert tape.instruction_count > 12000
    for thr in (None, 256):
        t2, got = _frames(device, text, 6, thr, times)
        assert t2.wide_threshold != NARROW_ONLY
        for (wc, wd, wr), (gc, gd, gr) in zip(want, got):
            assert_cells_equal(gc, wc)
            assert np.array_equal(gd, wd)
            assert np.array_equal(gr, wr)


@pytest.mark.gpu
def test_batch_autotune_scales_thresholds_and_keeps_results(device):
    texts = [scenes.csg(40, 21 + k, 0.8) for k in range(4)]
    tapes = [Tape.from_llvm_ir(device, t) for t in texts]
    base = [t.wide_threshold for t in tapes]
    sc = [Scene(device, t, api.default_params(localsubdiv=6)) for t in tapes]
    r = api.batch_autotune(device, [(s, 0.1 * k) for k, s in enumerate(sc)], frames=2)
    assert [m for m, _ in r["trials"]] == [1, 2, 4, 8]
    assert r["scale"] in (1, 2, 4, 8)
    for t, b in zip(tapes, base):
        assert t.wide_threshold == (NARROW_ONLY if b == NARROW_ONLY else b * r["scale"])
    # left reset, and the batch gives each scene's plain results
    res = api.run_batch(device, [(s, 0.1 * k, float("nan"), None) for k, s in enumerate(sc)])
    assert all(x["stats"].error_flags == 0 for x in res)
    for k, (text, s) in enumerate(zip(texts, sc)):
        fresh = Scene(device, Tape.from_llvm_ir(device, text), api.default_params(localsubdiv=6))
        fresh.invert(0.1 * k)
        assert_cells_equal(s.cells(), fresh.cells())
