"""Octree set inversion on the GPU against the CPU oracle, cell by cell.

Every cell of the resident octree (keyed by level and integer coordinates,
never by pool index) must carry the same classification f, evaluation time
t, accumulated time_err, fast flag, children flag, bounds and normal as the
oracle's restatement of compute.wgsl `main`, frame after frame, with tape
pruning on and off (pruning must never change a result).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from conftest import assert_cells_equal
from golden.make_golden import load_tape
from temporalsetinversion_b200 import Scene, Tape, _native as N, api, scenes

COUNTERS = ["parents_expanded", "cells_evaluated", "cells_reverse", "cells_skipped", "cells_ambiguous",
            "cells_empty", "cells_full", "cells_enqueued", "cells_reused"]


def _gen(fn, *a):
    return ("gen", fn, a)


CASES = {
    "spheres16_L6": (_gen(scenes.spheres16, 0), dict(localsubdiv=6, pointsample=0), [0.0, 1 / 60, 2 / 60, 3 / 60]),
    "spheres16_L7_point": (_gen(scenes.spheres16, 0), dict(localsubdiv=7, pointsample=1), [0.0, 0.02, 0.04]),
    "csg24_lipschitz": (_gen(scenes.csg, 24, 3, 0.9), dict(localsubdiv=6, lipschitz_corrected=1, pointsample=1),
                        [0.0, 0.05, 0.1, 0.15, 0.2]),
    "csg64_reuse": (_gen(scenes.csg, 64, 5, 0.85), dict(localsubdiv=7, delta=0.05), [i / 60 for i in range(6)]),
    "csg64_time_backwards": (_gen(scenes.csg, 64, 6, 0.9), dict(localsubdiv=6), [0.5, 0.25, 0.75, 0.7]),
    "swept8": (_gen(scenes.swept, 8, 4), dict(localsubdiv=5, swept_volume=1), [0.25, 0.5, 0.75]),
    "cables_L6": (("tape", "cables"), dict(localsubdiv=6), [0.0, 1 / 60, 2 / 60]),
    "cradle_L6": (("tape", "cradle"), dict(localsubdiv=6), [0.0, 1 / 60, 2 / 60]),
    "piano_L6": (("tape", "piano"), dict(localsubdiv=6), [0.0, 1 / 60, 2 / 60]),
    "sponza_L6": (("tape", "sponza"), dict(localsubdiv=6), [0.0, 1 / 60, 2 / 60]),
    "sponza_L5_normals": (("tape", "sponza"), dict(localsubdiv=5, normal_viz=1), [0.0, 0.1]),
}


def tape_of(src):
    if src[0] == "gen":
        return api.IR.new(src[1](*src[2])).gpu_instructions
    return load_tape(src[1])


@pytest.mark.gpu
@pytest.mark.parametrize("pruning", [1, 0])
@pytest.mark.parametrize("case", sorted(CASES))
def test_invert_matches_oracle(device, case, pruning):
    src, params, times = CASES[case]
    tape = tape_of(src)
    p = api.default_params(pruning=pruning, **params)
    gs = Scene(device, Tape.upload(device, tape), p)
    os_ = oracle.Scene(tape, p)
    for t in times:
        sg = gs.invert(t).as_dict()
        so = os_.invert(t)
        for k in COUNTERS:
            assert sg[k] == so[k], "t=%g %s: gpu %d oracle %d" % (t, k, sg[k], so[k])
        assert_cells_equal(gs.cells(), os_.cells())


@pytest.mark.gpu
def test_reset_is_first_eval(device):
    tape = tape_of(CASES["spheres16_L6"][0])
    p = api.default_params(localsubdiv=6, pointsample=0)
    gs = Scene(device, Tape.upload(device, tape), p)
    gs.invert(0.0)
    gs.invert(0.1)
    gs.reset()
    a = gs.invert(0.2).as_dict()
    fresh = Scene(device, Tape.upload(device, tape), p)
    b = fresh.invert(0.2).as_dict()
    for k in COUNTERS:
        assert a[k] == b[k]
    assert_cells_equal(gs.cells(), fresh.cells())


@pytest.mark.gpu
def test_llvm_ir_entry_equals_upload(device):
    text = scenes.csg(16, 9)
    p = api.default_params(localsubdiv=6)
    a = Scene(device, Tape.from_llvm_ir(device, text), p)
    b = Scene(device, Tape.upload(device, api.IR.new(text).gpu_instructions), p)
    for t in (0.0, 0.05):
        a.invert(t)
        b.invert(t)
    assert_cells_equal(a.cells(), b.cells())


@pytest.mark.gpu
def test_pruning_reduces_work(device):
    text = scenes.csg(128, 4)
    tape = api.IR.new(text).gpu_instructions
    on = Scene(device, Tape.upload(device, tape), api.default_params(localsubdiv=8, pruning=1))
    off = Scene(device, Tape.upload(device, tape), api.default_params(localsubdiv=8, pruning=0))
    s_on, s_off = on.invert(0.0), off.invert(0.0)
    assert s_on.cells_evaluated == s_off.cells_evaluated
    assert s_on.instr_forward * 2 < s_off.instr_forward
    assert s_off.instr_forward == s_off.instr_full_equiv
    assert_cells_equal(on.cells(), off.cells())


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["spheres16_L6", "csg64_reuse", "sponza_L6"])
def test_leaf_keys_match_oracle(device, case):
    """The leaf key set (cells with f <= 0 and no children, what the tracer
    can hit) equals the oracle's after every frame."""
    src, params, times = CASES[case]
    tape = tape_of(src)
    p = api.default_params(**params)
    gs = Scene(device, Tape.upload(device, tape), p)
    os_ = oracle.Scene(tape, p)
    for t in times:
        gs.invert(t)
        os_.invert(t)
        oc = os_.cells()
        want = oc[(oc["has_children"] == 0) & (oc["f"] <= 0)]
        want = {(int(c["level"]), int(c["ix"]), int(c["iy"]), int(c["iz"])) for c in want}
        got = {tuple(int(v) for v in row) for row in gs.leaves()}
        assert got == want, "t=%g: %d leaves, oracle %d" % (t, len(got), len(want))


@pytest.mark.gpu
def test_snapshot_restore_continues_exactly(device):
    """A scene restored from a snapshot into a fresh scene (same tape and
    parameters) continues frame for frame like the original."""
    src, params, times = CASES["csg64_reuse"]
    tape = tape_of(src)
    p = api.default_params(**params)
    a = Scene(device, Tape.upload(device, tape), p)
    for t in times[:3]:
        a.invert(t)
    blob = a.snapshot()
    b = Scene(device, Tape.upload(device, tape), p)
    b.restore(blob)
    assert_cells_equal(b.cells(), a.cells())
    for t in times[3:]:
        sa, sb = a.invert(t).as_dict(), b.invert(t).as_dict()
        for k in COUNTERS:
            assert sa[k] == sb[k]
        assert_cells_equal(b.cells(), a.cells())
    other = Scene(device, Tape.upload(device, tape), api.default_params(**dict(params, delta=0.02)))
    with pytest.raises(Exception):
        other.restore(blob)  # other parameters


@pytest.mark.gpu
def test_async_inversions_equal_plain(device):
    """Frames queued without waiting (inversion and traced frame) give the
    plain calls' octrees, counters and frames."""
    src, params, times = CASES["csg64_reuse"]
    tape = tape_of(src)
    p = api.default_params(**params)
    a = Scene(device, Tape.upload(device, tape), p)
    b = Scene(device, Tape.upload(device, tape), p)
    cam = scenes.camera_look_at((0.4, 0.8, 2.4))
    frames = [np.zeros((48, 64, 4), np.float32) for _ in times]
    want = []
    for t, buf in zip(times, frames):
        a.invert_async(t)
        a.trace_async(api.make_uniforms(cam, (64, 48), t), buf)
        sb = b.invert(t)
        want.append(b.trace(api.make_uniforms(cam, (64, 48), t), depth=False, normal=False)["rgba"])
    sa = a.invert_wait()
    a.trace_wait()
    for k in COUNTERS:
        assert getattr(sa, k) == getattr(sb, k), k
    assert_cells_equal(a.cells(), b.cells())
    for got, exp in zip(frames, want):
        assert np.array_equal(got, exp)


@pytest.mark.gpu
def test_async_inversion_reports_pool_exhaustion(device):
    tape = Tape.from_llvm_ir(device, scenes.spheres16(0))
    tiny = Scene(device, tape, api.default_params(localsubdiv=7), voxel_capacity=64)
    tiny.invert_async(0.0)
    tiny.invert_async(1 / 60)
    with pytest.raises(N.TsiError) as e:
        tiny.invert_wait()
    assert e.value.status == 4  # TSI_ERR_OOM
    ok = Scene(device, tape, api.default_params(localsubdiv=5))
    ok.invert_async(0.0)
    assert ok.invert_wait().cells_evaluated > 0


def _many_live(n: int, seed: int) -> str:
    """n moving spheres whose distances are all computed before a sequential
    min reduces them, so n values are live at once: a tape of more than n
    interval registers."""
    rng = np.random.default_rng(seed)
    b = scenes.IRBuilder()
    t2 = b.mul(b.T, 6.2831855)
    d = []
    for _ in range(n):
        c = rng.uniform(-0.7, 0.7, 3)
        m = b.mul(b.sin(b.add(t2, float(rng.uniform(0, 6.28)))), 0.1)
        q = [b.sub(v, b.add(m, float(ci))) for v, ci in zip((b.X, b.Y, b.Z), c)]
        s = b.add(b.add(b.mul(q[0], q[0]), b.mul(q[1], q[1])), b.mul(q[2], q[2]))
        d.append(b.sub(b.sqrt(s), float(rng.uniform(0.05, 0.15))))
    acc = d[0]
    for v in d[1:]:
        acc = b.min(acc, v)
    return b.text(acc)


@pytest.mark.gpu
def test_tape_beyond_pruning_registers_matches_oracle(device):
    """A tape with more live values than pruning handles (64 registers) runs
    unpruned, reports so in its counters, and still equals the oracle."""
    text = _many_live(70, 3)
    tape = api.IR.new(text).gpu_instructions
    t = Tape.upload(device, tape)
    assert t.registers > 64
    p = api.default_params(localsubdiv=6, pruning=1)
    gs = Scene(device, t, p)
    os_ = oracle.Scene(tape, p)
    unpruned = 0
    for tm in (0.0, 1 / 60, 2 / 60):
        st = gs.invert(tm)
        sg = st.as_dict()
        so = os_.invert(tm)
        for k in COUNTERS:
            assert sg[k] == so[k], "t=%g %s: gpu %d oracle %d" % (tm, k, sg[k], so[k])
        assert_cells_equal(gs.cells(), os_.cells())
        unpruned += st.cells_unpruned_regs
    assert unpruned > 0

