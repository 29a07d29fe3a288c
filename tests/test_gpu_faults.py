"""Failure detection without a GPU fault: exhausted pools and work lists come
back as error statuses from the host API and the device stays usable.  The
reference silently drops work in both cases (compute.wgsl:3159-3161 `enqueue`
returns false and its callers ignore it, 3537/4024/4041)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import assert_cells_equal
from temporalsetinversion_b200 import Device, Scene, Tape, _native as N, api, scenes


@pytest.mark.gpu
def test_voxel_pool_exhaustion_is_reported(device):
    tape = Tape.from_llvm_ir(device, scenes.spheres16(0))
    tiny = Scene(device, tape, api.default_params(localsubdiv=7), voxel_capacity=64)
    with pytest.raises(N.TsiError) as e:
        tiny.invert(0.0)
    assert e.value.status == 4  # TSI_ERR_OOM
    ok = Scene(device, tape, api.default_params(localsubdiv=5))
    st = ok.invert(0.0)
    assert st.cells_evaluated > 0 and st.error_flags == 0


@pytest.mark.gpu
def test_graph_replay_reports_pool_exhaustion(device):
    """A graph replay that runs out of voxels reports it at the wait, like
    the plain call, and a replay after a reset of a large enough scene works."""
    tape = Tape.from_llvm_ir(device, scenes.spheres16(0))
    tiny = Scene(device, tape, api.default_params(localsubdiv=7), voxel_capacity=64)
    ok = Scene(device, tape, api.default_params(localsubdiv=5))
    g = api.BatchGraph(device, [(tiny, 0.0, float("nan"), None), (ok, 0.0, float("nan"), None)])
    try:
        g.launch([0.0, 0.0])
        with pytest.raises(N.TsiError) as e:
            g.wait()
        assert e.value.status == 4  # TSI_ERR_OOM
    finally:
        g.close()
    g = api.BatchGraph(device, [(ok, 0.1, float("nan"), None)])
    try:
        ok.reset()
        g.launch([0.1])
        st = g.wait()
        assert st.error_flags == 0 and st.cells_evaluated > 0
    finally:
        g.close()


@pytest.mark.gpu
def test_batch_wider_than_one_launch_reports_every_chunk():
    """A batch of more scenes than one launch takes runs as consecutive
    launch sequences; an exhausted pool in the FIRST chunk is still reported
    (status and that request's error bits), and every other request's
    counters are its own."""
    with Device(max_scenes_per_launch=4) as dev:
        tape = Tape.from_llvm_ir(dev, scenes.spheres16(0))
        tiny = Scene(dev, tape, api.default_params(localsubdiv=7), voxel_capacity=64)
        rest = [Scene(dev, tape, api.default_params(localsubdiv=5)) for _ in range(6)]
        alone = Scene(dev, tape, api.default_params(localsubdiv=5))
        want = alone.invert(0.0)
        reqs = [(tiny, 0.0, float("nan"), None)] + [(s, 0.0, float("nan"), None) for s in rest]
        with pytest.raises(N.TsiError) as e:
            api.run_batch(dev, reqs)
        assert e.value.status == 4  # TSI_ERR_OOM, from the first of two chunks
        out = [N.Stats() for _ in reqs]
        arr = (N.Request * len(reqs))()
        for i, (sc, t, t0, _) in enumerate(reqs):
            sc.reset()
            arr[i].scene, arr[i].time, arr[i].t0_or_nan = sc.handle, t, t0
            arr[i].stats = C.pointer(out[i])
        assert dev.lib.tsi_batch_run(dev.handle, arr, len(reqs)) == 4
        assert out[0].error_flags != 0
        for st in out[1:]:
            assert st.error_flags == 0
            assert (st.cells_evaluated, st.cells_enqueued, st.voxels_live) == (
                want.cells_evaluated, want.cells_enqueued, want.voxels_live)


@pytest.mark.gpu
def test_trace_async_rejects_mismatched_frame(device):
    tape = Tape.from_llvm_ir(device, scenes.spheres16(0))
    s = Scene(device, tape, api.default_params(localsubdiv=4))
    s.invert(0.0)
    u = api.make_uniforms(scenes.camera_look_at((0.4, 0.8, 2.4)), (32, 16), 0.0)
    img = N.Image(16, 16, None, None, None)
    assert device.lib.tsi_scene_trace_async(s.handle, C.byref(u), C.byref(img)) == 10  # TSI_ERR_BUFFER_TOO_SMALL
    rgba = np.zeros((16, 32, 4), np.float32)
    s.trace_async(u, rgba)
    s.trace_wait()
    assert np.array_equal(rgba, s.trace(u, depth=False, normal=False)["rgba"])


@pytest.mark.gpu
def test_work_list_overflow_is_reported():
    with Device(work_item_capacity=16) as dev:
        tape = Tape.from_llvm_ir(dev, scenes.spheres16(0))
        s = Scene(dev, tape, api.default_params(localsubdiv=6))
        with pytest.raises(N.TsiError) as e:
            s.invert(0.0)
        assert e.value.status == 5  # TSI_ERR_QUEUE_FULL
        s2 = Scene(dev, tape, api.default_params(localsubdiv=2))
        assert s2.invert(0.0).cells_evaluated > 0


@pytest.mark.gpu
def test_bad_opcode_and_bad_tapes_rejected(device):
    tape = api.IR.new(scenes.spheres16(0)).gpu_instructions.copy()
    bad = tape.copy()
    bad[10]["opcode_uses"] = (31 | (1 << 14)) << 16 | 1  # opcode 31 does not exist
    with pytest.raises(N.TsiError) as e:
        Tape.upload(device, bad)
    assert e.value.status == 7  # TSI_ERR_BAD_OPCODE
    fwd = tape.copy()
    fwd[10]["larg_rarg"] = (12 << 16) | 11  # reads slots not yet computed
    fwd[10]["opcode_uses"] = (5 << 16) | 1
    with pytest.raises(N.TsiError) as e:
        Tape.upload(device, fwd)
    assert e.value.status == 1
    with pytest.raises(N.TsiError) as e:
        Tape.from_llvm_ir(device, "define float @_Z1fffff(float %0) {\n  %5 = fcmp olt float %0, %1\n}\n")
    assert e.value.status == 2  # TSI_ERR_PARSE
    # the device is still usable
    s = Scene(device, Tape.upload(device, tape), api.default_params(localsubdiv=4))
    assert s.invert(0.0).cells_evaluated > 0


def _serial_chain(n: int) -> str:
    """A sphere followed by a chain of n dependent multiply-adds: a long tape
    with no parallelism, which stays on the one-warp path."""
    b = scenes.IRBuilder()
    v = b.add(b.add(b.mul(b.X, b.X), b.mul(b.Y, b.Y)), b.mul(b.Z, b.Z))
    v = b.add(v, b.mul(b.T, 0.1))
    for _ in range(n):
        v = b.sub(b.mul(v, 1.0001), 0.0001)
    return b.text(b.sub(v, 0.25))


@pytest.mark.gpu
def test_log_arena_exhaustion_is_reported():
    with Device(log_arena_bytes=1 << 16) as dev:
        # ~1.2k dependent instructions: the operand log outgrows a warp's slice
        text = _serial_chain(600)
        s = Scene(dev, Tape.from_llvm_ir(dev, text), api.default_params(localsubdiv=3))
        with pytest.raises(N.TsiError) as e:
            for t in (0.0, 0.02):  # the second frame runs reverse AD on the long root tape
                s.invert(t)
        assert e.value.status == 4
        s2 = Scene(dev, Tape.from_llvm_ir(dev, scenes.spheres16(0)), api.default_params(localsubdiv=4))
        assert s2.invert(0.0).cells_evaluated > 0


@pytest.mark.gpu
def test_hbm_budget_admits_scenes_and_frames():
    """Scenes and frame buffers are admitted against the context's HBM
    budget; an idle scene evicted to host memory (snapshot, destroy) and
    readmitted (create, restore) continues frame for frame."""
    text = scenes.spheres16(0)
    p = api.default_params(localsubdiv=6)
    with Device() as probe:
        s = Scene(probe, Tape.from_llvm_ir(probe, text), p, voxel_capacity=1 << 16)
        per = probe.scenes_bytes()
        assert per == s.device_bytes() > 0
        s.close()
    with Device(hbm_budget_bytes=2 * per + per // 2) as dev:
        tape = Tape.from_llvm_ir(dev, text)
        a = Scene(dev, tape, p, voxel_capacity=1 << 16)
        b = Scene(dev, tape, p, voxel_capacity=1 << 16)
        assert dev.scenes_bytes() == 2 * per
        with pytest.raises(N.TsiError) as e:
            Scene(dev, tape, p, voxel_capacity=1 << 16)
        assert e.value.status == 4  # TSI_ERR_OOM
        a.invert(0.0)
        with pytest.raises(N.TsiError) as e:  # a frame buffer of ~4 scenes' size does not fit
            a.trace(api.make_uniforms(scenes.camera_look_at((0.3, 0.6, 2.5)), (2048, 2048), 0.0))
        assert e.value.status == 4
        # evict a (its octree to the host), admit c, readmit a
        a.invert(1 / 60)
        blob = a.snapshot()
        a.close()
        c = Scene(dev, tape, p, voxel_capacity=1 << 16)
        c.close()
        a2 = Scene(dev, tape, p, voxel_capacity=1 << 16)
        a2.restore(blob)
        st = a2.invert(2 / 60)
        for t in (0.0, 1 / 60, 2 / 60):  # b lived through the same frames resident
            sb = b.invert(t)
        assert st.error_flags == 0 and st.cells_evaluated == sb.cells_evaluated
        assert_cells_equal(a2.cells(), b.cells())
