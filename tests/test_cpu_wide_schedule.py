"""The bundled (wide) tape form, checked on the host: every instruction
scheduled once, after its operands; at most 256 slots per bundle (one block
executes a bundle, one thread per slot) in groups of 32 slots (one warp
each) of one handler, the lanes a group leaves free holding padding slots;
every value in its own SSA slot; and contribution records that let a value
with several users sum its sensitivity in reverse program order (the order
of the sequential reverse pass, which fixes the rounding) wherever its users
were scheduled.  No device needed."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from golden.make_golden import load_tape
from temporalsetinversion_b200 import _native as N, api, scenes

NONE = 0xFFFFFFFF


def wide(tape: np.ndarray):
    lib = N.load()
    arr = np.ascontiguousarray(tape, dtype=api.GPU_INSTR_DTYPE)
    ptr = arr.ctypes.data_as(C.POINTER(N.GPUInstruction))
    info, nb = N.TapeInfo(), C.c_uint32(0)
    N.check(lib.tsi_compile_wide_gpu_instructions(ptr, len(arr), None, 0, None, 0, C.byref(info), C.byref(nb)), "wide")
    bundles = np.zeros(nb.value * 2, np.uint32)
    N.check(lib.tsi_compile_wide_gpu_instructions(ptr, len(arr), None, 0, bundles.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                  len(bundles), C.byref(info), C.byref(nb)), "wide")
    n_slots = int(bundles[-2]) + int(bundles[-1])  # padding slots included
    slots = np.zeros(n_slots * 12, np.uint32)
    N.check(lib.tsi_compile_wide_gpu_instructions(
        ptr, len(arr), slots.ctypes.data_as(C.POINTER(C.c_uint32)), len(slots),
        bundles.ctypes.data_as(C.POINTER(C.c_uint32)), len(bundles), C.byref(info), C.byref(nb)), "wide")
    return slots.reshape(n_slots, 12), bundles.reshape(-1, 2), info


PAD = 63


CASES = {
    "cables": lambda: load_tape("cables"),
    "sponza": lambda: load_tape("sponza"),
    "spheres16": lambda: api.IR.new(scenes.spheres16(0)).gpu_instructions,
    "swept8": lambda: api.IR.new(scenes.swept(8, 4)).gpu_instructions,
    "csg64": lambda: api.IR.new(scenes.csg(64, 5, 0.85)).gpu_instructions,
    "csg256": lambda: api.IR.new(scenes.csg(256, 1)).gpu_instructions,
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_wide_schedule_invariants(case):
    tape = CASES[case]()
    n = len(tape)
    slots, bundles, info = wide(tape)
    assert info.registers == n  # one value slot per SSA value
    bundle_of = {a: -1 for a in range(4)}
    seen = np.zeros(n, bool)
    next_first = 0
    for k, (first, count) in enumerate(bundles):
        first, count = int(first), int(count)
        assert first == next_first and 1 <= count <= 256
        next_first = first + count
        group = slots[first:first + count]
        for w in range(0, count, 32):
            warp = group[w:w + 32]
            hs = {int(s[0]) & 63 for s in warp} - {PAD}
            assert len(hs) == 1, "bundle %d warp %d mixes handlers %s" % (k, w // 32, hs)
            live = [int(s[0]) & 63 != PAD for s in warp]
            assert live[0] and live == sorted(live, reverse=True), "padding only after a group's slots"
        for s in group:
            if int(s[0]) & 63 == PAD:
                assert list(map(int, s[4:12])) == [0, NONE, NONE, NONE, NONE, NONE, NONE, 0]
                continue
            j = int(s[4])
            assert int(s[0]) >> 8 == j
            assert not seen[j]
            seen[j] = True
            bundle_of[j] = k
    assert next_first == len(slots)
    assert seen[4:].all()
    users, rec = {}, {}
    slots = slots[(slots[:, 0] & 63) != PAD]
    for s in slots:
        j, a, b = int(s[4]), int(s[6]), int(s[7])
        h = int(s[0]) & 63
        assert int(s[1]) == (a if a != NONE else 0)
        if b != NONE:
            assert int(s[2]) == b
        if int(s[5]) != NONE:  # min/max: ordinal in the word the handler does not use
            assert int(s[3]) == int(s[5]) if b != NONE else int(s[2]) == int(s[5])
        for v in {a, b} - {NONE}:
            assert bundle_of[v] < bundle_of[j], "slot %d runs before its operand %d" % (j, v)
            users.setdefault(v, []).append(j)
        if a != NONE:
            rec[(j, a)] = int(s[8])
        if b != NONE:
            assert b != a or int(s[9]) == int(s[8])
            rec[(j, b)] = int(s[9])
    first = {int(s[4]): (int(s[10]), int(s[11])) for s in slots}
    taken = set()
    for v, us in users.items():
        if len(us) == 1:
            assert rec[(us[0], v)] == NONE and first.get(v, (NONE, 0))[1] == 0
            continue
        if v >= 4:
            base, count = first[v]
            assert count == len(us)
            # records run last user first
            assert [rec[(j, v)] for j in sorted(us, reverse=True)] == list(range(base, base + count))
        for j in us:
            assert rec[(j, v)] not in taken
            taken.add(rec[(j, v)])
    assert len(taken) == info.reserved  # contribution records per cell


@pytest.mark.parametrize("case,steps", [("csg256", 32), ("csg64", 29), ("cables", 44), ("spheres16", 27)])
def test_wide_schedule_length(case, steps):
    """Warp groups of different handlers share a step, so a tape takes about
    as many bundle steps as its dependency depth (csg256: 4693 instructions
    of depth 31 in 32 steps; cables: depth 44)."""
    _, bundles, _ = wide(CASES[case]())
    assert len(bundles) <= steps


# handlers the device evaluates inline (the rest run out of line)
INLINE = {0, 1, 2, 3, 4, 6, 7, 12, 13, 14, 16, 17, 21, 22, 25, 26, 31}


@pytest.mark.parametrize("case,bound", [("swept64", 4), ("csg256", 1), ("csg64", 1), ("spheres16", 1)])
def test_out_of_line_handlers_gather(case, bound):
    """Elementary functions and divisions cost several ordinary steps each,
    so the schedule gathers them: they wait while they have slack and a
    step that takes one takes all its ready instructions (the rotating
    swept scene's 64 sines and 64 cosines fill 4 steps, not 17)."""
    tape = (api.IR.new(scenes.swept(64, 2)).gpu_instructions if case == "swept64" else CASES[case]())
    slots, bundles, _ = wide(tape)
    steps = 0
    for first, count in bundles:
        hs = {int(s[0]) & 63 for s in slots[int(first):int(first) + int(count)]} - {PAD}
        steps += bool(hs - INLINE)
    assert steps <= bound, steps

