"""Test helper: the nearest-depth composite of subtree frames restated in
numpy (the checker of tsi_frames_composite, tsi_frame_keep_nearest and
split.combine_ranks).  Key per pixel and part: the depth's bits in the high
word for a hit (depth >= 0), 0x7fffffff for a miss, the subtree index in
the low word; the least key wins."""
from __future__ import annotations

import numpy as np

import oracle
from temporalsetinversion_b200 import split


def keys(depth: np.ndarray, sid: int) -> np.ndarray:
    hi = np.where(depth >= 0, depth.view(np.uint32) & np.uint32(0x7FFFFFFF), np.uint32(0x7FFFFFFF))
    return ((hi.astype(np.uint64) << np.uint64(32)) | np.uint64(sid)).astype(np.int64)


def composite(parts: list, ids: list) -> dict:
    """parts: dicts of rgba (h, w, 4), depth (h, w), normal (h, w, 3)."""
    k = np.stack([keys(p["depth"], i) for p, i in zip(parts, ids)])
    win = k.argmin(axis=0)
    out = {"key": k.min(axis=0)}
    for name in ("rgba", "depth", "normal"):
        stack = np.stack([p[name] for p in parts])
        out[name] = np.take_along_axis(stack, win[None, ..., None] if stack.ndim == 4 else win[None], axis=0)[0]
    return out


def keep_nearest(frame: dict, global_key: np.ndarray) -> None:
    lost = frame["key"] != global_key
    for name in ("rgba", "depth", "normal"):
        frame[name][lost] = 0.0


def oracle_parts(tape, params, level: int, ids: list, times: list, uniforms) -> list:
    """Oracle scenes of subtrees `ids`, inverted at `times`, traced once."""
    out = []
    for k in ids:
        s = oracle.Scene(tape, split.subtree_params(params, level, k))
        for t in times:
            s.invert(t)
        out.append(s.trace(uniforms))
    return out
