"""One animation split at the root on the device (temporalsetinversion_b200.split):
every subtree scene against the oracle's scene of the same subtree (cells
and frames bit for bit, frame after frame), tsi_frames_composite against the
numpy composite, and two ranks' frames combined by keep-nearest and an
integer sum (what split.combine_ranks does over NCCL) against the one-rank
composite, bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import split_ref
from conftest import assert_cells_equal
from temporalsetinversion_b200 import Tape, _native as N, api, scenes, split

TIMES = [0.0, 1.0 / 60.0, 2.0 / 60.0]


def _host(fb: dict) -> dict:
    return {k: v.cpu().numpy().copy() for k, v in fb.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("level", [1, 2])
def test_subtree_scenes_and_composite_match_oracle(device, level):
    import torch
    text = scenes.csg(24, 3, 0.9)
    tape = api.IR.new(text).gpu_instructions
    p = api.default_params(localsubdiv=7, lipschitz_corrected=1)
    sp = split.SubtreeSplit(device, Tape.upload(device, tape), p, level=level, voxel_capacity=1 << 18)
    parts = [oracle.Scene(tape, split.subtree_params(p, level, k)) for k in sp.ids]
    w, h = 160, 90
    u = api.make_uniforms(scenes.camera_look_at((1.2, 0.8, 1.4)), (w, h), 0.0)
    for t in TIMES:
        u.time = t
        fb, stats = sp.frame(t, u)
        got = _host(fb)
        frames = []
        for k, (s, o) in enumerate(zip(sp.scenes, parts)):
            so = o.invert(t)
            # one fused launch sequence; each part's counters are its own
            assert (stats[k].cells_evaluated, stats[k].cells_reused) == (so["cells_evaluated"], so["cells_reused"])
            assert_cells_equal(s.cells(), o.cells())
            g, r = s.image(w, h), o.trace(u)
            for key in ("rgba", "depth", "normal"):
                assert g[key].tobytes() == r[key].tobytes(), (t, key)
            frames.append(r)
        want = split_ref.composite(frames, sp.ids)
        assert (want["depth"] >= 0).sum() > 1000
        for key in ("rgba", "depth", "normal", "key"):
            assert got[key].tobytes() == want[key].tobytes(), (t, key)
        assert torch.all(fb["key"] > 0)  # positive as int64
    sp.close()


@pytest.mark.gpu
def test_two_ranks_combine_to_the_one_rank_composite(device):
    """Ranks 0 and 1 of 2 (subtrees even and odd, their scenes on this one
    device, run one after the other): the elementwise MIN of their keys,
    keep-nearest on each and the sum of their bits as int32 equal the
    composite of one rank holding all eight subtrees."""
    import torch
    tape = Tape.upload(device, api.IR.new(scenes.csg(24, 3, 0.9)).gpu_instructions)
    p = api.default_params(localsubdiv=7, lipschitz_corrected=1)
    one = split.SubtreeSplit(device, tape, p, level=1, voxel_capacity=1 << 18)
    ranks = [split.SubtreeSplit(device, tape, p, level=1, rank=r, world=2, voxel_capacity=1 << 18) for r in range(2)]
    u = api.make_uniforms(scenes.camera_look_at((1.2, 0.8, 1.4)), (192, 108), 0.0)
    for t in TIMES:
        u.time = t
        want = _host(one.frame(t, u)[0])
        fbs = [{k: v.clone() for k, v in r.frame(t, u)[0].items()} for r in ranks]
        gkey = torch.minimum(fbs[0]["key"], fbs[1]["key"])
        for r, fb in zip(ranks, fbs):
            r.keep_nearest(fb, gkey)
        for key in ("rgba", "depth", "normal"):
            merged = fbs[0][key].view(torch.int32) + fbs[1][key].view(torch.int32)
            assert merged.cpu().numpy().tobytes() == want[key].view(np.int32).tobytes(), (t, key)
        assert gkey.cpu().numpy().tobytes() == want["key"].tobytes()
    for s in [one] + ranks:
        s.close()


@pytest.mark.gpu
def test_composite_rejects_mismatched_parts(device):
    import ctypes as C

    import torch
    tape = Tape.upload(device, api.IR.new(scenes.spheres16(0)).gpu_instructions)
    p = api.default_params(localsubdiv=5)
    sp = split.SubtreeSplit(device, tape, p, level=1, voxel_capacity=1 << 16)
    u = api.make_uniforms(scenes.camera_look_at((0.5, 0.5, 1.3)), (64, 36), 0.0)
    fb, _ = sp.frame(0.0, u)
    # a frame of another size
    other = sp.buffers(32, 18)
    with pytest.raises(N.TsiError) as e:
        sp.composite(other)
    assert e.value.status == 10  # TSI_ERR_BUFFER_TOO_SMALL
    fb = sp.buffers(64, 36)
    # the same subtree twice
    handles = (C.c_void_p * 2)(sp.scenes[0].handle.value, sp.scenes[1].handle.value)
    ids = (C.c_uint32 * 2)(3, 3)
    out = split.frame_struct(fb, 64, 36)
    assert device.lib.tsi_frames_composite(device.handle, handles, ids, 2, C.byref(out)) == 1
    # misaligned rgba
    bad = dict(fb, rgba=torch.empty(64 * 36 * 4 + 1, dtype=torch.float32, device=fb["rgba"].device)[1:])
    assert device.lib.tsi_frames_composite(device.handle, handles, (C.c_uint32 * 2)(0, 1), 2,
                                           C.byref(split.frame_struct(bad, 64, 36))) == 1
    sp.close()
