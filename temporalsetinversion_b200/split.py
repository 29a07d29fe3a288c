"""One animation split at the root over several scenes and GPUs.

The reference keeps one octree per device and expands its root every frame
(buf_main, compute.wgsl:4690-4708); the root's subtrees never read one
another, so the animation can be cut at `level` into 8**level subtrees,
each inverted as a scene of its own (tsi_params_subtree: the root box is
that cell's box, bit for bit the full octree's bounds and epsilon).  Each
part is traced over the whole image and the frames are composited by
nearest depth:

* on one GPU, tsi_frames_composite picks per pixel the part with the least
  key (depth bits << 32 | subtree index; misses sort after every hit);
* across GPUs (one process per GPU, this module's combine_ranks), a MIN
  all-reduce of the keys over int64, then every rank zeroes the pixels it
  did not win (tsi_frame_keep_nearest) and a SUM reduce of the pixels' bits
  as int32 gathers the composite on one rank, bit for bit (every pixel has
  exactly one winner; the others add zero bits).

Subtrees are dealt to ranks cyclically, so each rank's share is spread over
the scene.  The composite's depth and normal of a hit are those of the
winning part's ray; the tracer's darkening only counts the nodes of that
part, and an all-miss pixel takes the miss colour of subtree 0.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N
from .api import Device, Scene, Tape

__all__ = ["subtree_params", "subtree_ids", "SubtreeSplit", "combine_ranks", "KEY_MISS"]

KEY_MISS = 0x7FFFFFFF  # high word of a miss's key
COMPOSITE_MAX = 64     # TSI_COMPOSITE_MAX


def subtree_params(params: N.Params, level: int, index: int) -> N.Params:
    """`params` with the root box of subtree `index` = ix + n (iy + n iz),
    n = 2**level (tsi_params_subtree)."""
    out = N.Params()
    N.check(N.load().tsi_params_subtree(C.byref(params), int(level), int(index), C.byref(out)), "tsi_params_subtree")
    return out


def subtree_ids(level: int, rank: int = 0, world: int = 1) -> list:
    """The subtrees of `rank` among `world` parts: every world-th index."""
    if not 0 <= rank < world:
        raise ValueError("rank %d outside world %d" % (rank, world))
    return list(range(rank, 8 ** level, world))


def subtree_cell_keys(cells: np.ndarray, level: int, index: int) -> np.ndarray:
    """A part's cells keyed like the full octree's: (level + l, (sx << l) + ix, ...)."""
    n = 1 << level
    sx, sy, sz = index % n, (index // n) % n, index // (n * n)
    out = cells.copy()
    lv = cells["level"].astype(np.uint64)
    out["level"] = cells["level"] + level
    out["ix"] = ((np.uint64(sx) << lv) + cells["ix"]).astype(np.uint32)
    out["iy"] = ((np.uint64(sy) << lv) + cells["iy"]).astype(np.uint32)
    out["iz"] = ((np.uint64(sz) << lv) + cells["iz"]).astype(np.uint32)
    return out


class SubtreeSplit:
    """This rank's share of one animation cut at `level`: one scene per
    owned subtree on `device`, inverted together (tsi_batch_run, one fused
    launch sequence), traced, and composited on the device."""

    def __init__(self, device: Device, tape: Tape, params: N.Params, level: int = 1, rank: int = 0, world: int = 1,
                 voxel_capacity: int = 0):
        self.device, self.level = device, level
        self.ids = subtree_ids(level, rank, world)
        if not 0 < len(self.ids) <= COMPOSITE_MAX:
            raise ValueError("a rank holds 1 to %d subtrees (has %d)" % (COMPOSITE_MAX, len(self.ids)))
        self.scenes = [Scene(device, tape, subtree_params(params, level, k), voxel_capacity) for k in self.ids]
        self._fb = None

    def close(self) -> None:
        for s in self.scenes:
            s.close()
        self.scenes = []
        self._fb = None

    def reset(self) -> None:
        for s in self.scenes:
            s.reset()

    def _run(self, time: float, t0: float, uniforms) -> list:
        n = len(self.scenes)
        reqs = (N.Request * n)()
        stats = [N.Stats() for _ in range(n)]
        for i, s in enumerate(self.scenes):
            reqs[i].scene = s.handle
            reqs[i].time = float(time)
            reqs[i].t0_or_nan = float(t0)
            reqs[i].stats = C.pointer(stats[i])
            if uniforms is not None:
                reqs[i].uniforms = C.pointer(uniforms)  # frames stay on the device (out = NULL)
        N.check(self.device.lib.tsi_batch_run(self.device.handle, reqs, n), "tsi_batch_run")
        return stats

    def invert(self, time: float, t0: float = math.nan) -> list:
        """Inverts every owned subtree at `time`; per-part tsi_stats."""
        return self._run(time, t0, None)

    def buffers(self, width: int, height: int) -> dict:
        """The composite's device buffers (torch tensors on this device),
        kept across frames of the same size."""
        import torch
        fb = self._fb
        if fb is None or fb["depth"].shape != (height, width):
            dev = torch.device("cuda", self.device.index)
            fb = {"rgba": torch.empty((height, width, 4), dtype=torch.float32, device=dev),
                  "depth": torch.empty((height, width), dtype=torch.float32, device=dev),
                  "normal": torch.empty((height, width, 3), dtype=torch.float32, device=dev),
                  "key": torch.empty((height, width), dtype=torch.int64, device=dev)}
            self._fb = fb
        return fb

    def frame(self, time: float, uniforms: N.Uniforms, t0: float = math.nan) -> tuple:
        """Inverts the owned subtrees at `time`, traces them with `uniforms`
        and composites them: (frame as device tensors rgba, depth, normal,
        key; per-part stats)."""
        import torch
        w, h = int(uniforms.resolution[0]), int(uniforms.resolution[1])
        fb = self.buffers(w, h)
        torch.cuda.current_stream(fb["depth"].device).synchronize()  # no earlier collective still reads them
        stats = self._run(time, t0, uniforms)
        self.composite(fb)
        return fb, stats

    def composite(self, fb: dict) -> None:
        """tsi_frames_composite of the owned parts' last frames into fb."""
        n = len(self.scenes)
        h, w = fb["depth"].shape
        handles = (C.c_void_p * n)(*[s.handle.value for s in self.scenes])
        ids = (C.c_uint32 * n)(*self.ids)
        out = frame_struct(fb, w, h)
        N.check(self.device.lib.tsi_frames_composite(self.device.handle, handles, ids, n, C.byref(out)),
                "tsi_frames_composite")

    def keep_nearest(self, fb: dict, global_key) -> None:
        """tsi_frame_keep_nearest: zero the pixels whose key is not the global one."""
        h, w = fb["depth"].shape
        out = frame_struct(fb, w, h)
        N.check(self.device.lib.tsi_frame_keep_nearest(self.device.handle, C.c_void_p(global_key.data_ptr()),
                                                       C.byref(out)), "tsi_frame_keep_nearest")

    def cells(self) -> np.ndarray:
        """Every part's cells keyed like the full octree's (the parts' roots,
        which the full octree holds as ordinary cells, excluded)."""
        parts = [subtree_cell_keys(s.cells(), self.level, k) for s, k in zip(self.scenes, self.ids)]
        cells = np.concatenate(parts)
        return cells[cells["level"] > self.level]


def frame_struct(fb: dict, width: int, height: int) -> N.FrameDevice:
    for name in ("rgba", "depth", "normal", "key"):
        if not fb[name].is_contiguous():
            raise ValueError("frame buffer %s is not contiguous" % name)
    return N.FrameDevice(width, height, fb["rgba"].data_ptr(), fb["depth"].data_ptr(), fb["normal"].data_ptr(),
                         fb["key"].data_ptr())


def combine_ranks(fb: dict, keep_nearest, group=None, dst: int = 0) -> dict | None:
    """Gathers the nearest-depth composite of every rank's frame `fb` on
    global rank `dst` (returned there; None elsewhere).  keep_nearest(fb, global_key)
    zeroes the pixels this rank did not win (SubtreeSplit.keep_nearest).
    Collectives: one MIN all-reduce of the int64 keys, one SUM reduce per
    output of its bits as int32.  fb is overwritten."""
    import torch
    import torch.distributed as dist
    gkey = fb["key"].clone()
    dist.all_reduce(gkey, op=dist.ReduceOp.MIN, group=group)
    if gkey.is_cuda:
        torch.cuda.current_stream(gkey.device).synchronize()
    keep_nearest(fb, gkey)
    for name in ("rgba", "depth", "normal"):
        dist.reduce(fb[name].view(torch.int32), dst, op=dist.ReduceOp.SUM, group=group)
    fb["key"].copy_(gkey)
    if fb["depth"].is_cuda:
        torch.cuda.current_stream(fb["depth"].device).synchronize()
    return fb if dist.get_rank() == dst else None
