"""Allocation-free box evaluation: tsi_tape_eval_boxes_static against
tsi_tape_eval_boxes on the same tape and boxes.

The static entry point keeps its scratch in a file-scope device array and
takes device pointers; this file is collected last so that it also runs after
every other GPU test has used (and grown) the context's allocating scratch.
Both entry points run the same kernel, so results are compared bit for bit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from temporalsetinversion_b200 import Tape, scenes
from temporalsetinversion_b200 import _native as N


def _boxes(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    lo = rng.uniform(-1.2, 1.2, (n, 4)).astype(np.float32)
    w = (rng.uniform(0, 1, (n, 4)) ** 2 * 0.6).astype(np.float32)
    w[rng.uniform(size=(n, 4)) < 0.15] = 0.0  # point intervals
    b = np.empty((n, 8), np.float32)
    b[:, 0::2], b[:, 1::2] = lo, (lo + w).astype(np.float32)
    return b


def _same(a: np.ndarray, b: np.ndarray) -> bool:
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def _static(lib, tape, boxes_t, out_t, rounding, reverse, stream):
    return lib.tsi_tape_eval_boxes_static(tape.handle, boxes_t.shape[0], C.c_void_p(boxes_t.data_ptr()), rounding,
                                          reverse, C.c_void_p(out_t.data_ptr()), C.c_void_p(stream))


@pytest.mark.gpu
def test_static_eval_matches_allocating_eval_twice(device):
    import torch

    lib = device.lib
    assert lib.tsi_static_scratch_bytes() == 16 << 20
    tape = Tape.from_llvm_ir(device, scenes.csg(48, 4, 0.9))
    per_box = 8 * tape.registers + 16 * tape.instruction_count
    n = min(1024, (16 << 20) // (per_box + 8) - 1)
    assert n >= 64
    side = torch.cuda.Stream()
    # (rounding, reverse, seed, stream): a caller's stream, then the tape
    # context's stream (NULL) for the call right after it
    cases = [(0, 1, 11, side), (0, 1, 12, None), (1, 0, 13, side), (1, 0, 14, None)]
    for rounding, reverse, seed, stream in cases:
        boxes = _boxes(n, seed)
        want = tape.eval_boxes(boxes, rounding_mode=rounding, reverse=bool(reverse))
        b = torch.from_numpy(boxes).cuda()
        out = torch.full((n, 10), float("nan"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        if stream is not None:
            N.check(_static(lib, tape, b, out, rounding, reverse, stream.cuda_stream), "tsi_tape_eval_boxes_static")
            stream.synchronize()
        else:
            N.check(_static(lib, tape, b, out, rounding, reverse, None), "tsi_tape_eval_boxes_static")
            N.check(lib.tsi_synchronize(device.handle), "tsi_synchronize")
        got = out.cpu().numpy()
        assert _same(got, want), "rounding %d reverse %d: %d boxes differ" % (
            rounding, reverse, int((~((got == want) | (np.isnan(got) & np.isnan(want)))).any(axis=1).sum()))


@pytest.mark.gpu
def test_static_eval_rejects_oversize_and_null(device):
    import torch

    lib = device.lib
    tape = Tape.from_llvm_ir(device, scenes.csg(48, 4, 0.9))
    n_over = 2 * (16 << 20) // (16 * tape.instruction_count) + 1  # about twice what the array holds
    b = torch.zeros((n_over, 8), dtype=torch.float32, device="cuda")
    out = torch.zeros((n_over, 10), dtype=torch.float32, device="cuda")
    assert _static(lib, tape, b, out, 0, 1, None) == 10  # TSI_ERR_BUFFER_TOO_SMALL, nothing launched
    assert b"static scratch" in lib.tsi_last_error()
    assert lib.tsi_tape_eval_boxes_static(tape.handle, 4, None, 0, 1, C.c_void_p(out.data_ptr()), None) == 1
    assert _static(lib, tape, b[:0], out, 0, 1, None) == 0  # n = 0: nothing to do
