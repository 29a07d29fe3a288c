"""The bundled (wide) tape form, checked on the host: every slot scheduled
once, after its operands, at most 256 slots and one handler per bundle
(one block executes a bundle, one thread per slot), every value in its own
SSA slot, and contribution records that let a value with several users sum
its sensitivity in reverse program order (the order of the sequential
reverse pass, which fixes the rounding) wherever its users were scheduled.
No device needed."""
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
    n_slots = len(arr) - 4
    slots = np.zeros(n_slots * 12, np.uint32)
    bundles = np.zeros(nb.value * 2, np.uint32)
    N.check(lib.tsi_compile_wide_gpu_instructions(
        ptr, len(arr), slots.ctypes.data_as(C.POINTER(C.c_uint32)), len(slots),
        bundles.ctypes.data_as(C.POINTER(C.c_uint32)), len(bundles), C.byref(info), C.byref(nb)), "wide")
    return slots.reshape(n_slots, 12), bundles.reshape(-1, 2), info


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
    for k, (first, word) in enumerate(bundles):
        count, h = int(word) & 0xFFFF, int(word) >> 16
        assert 1 <= count <= 256
        group = slots[first:first + count]
        assert {int(s[0]) & 63 for s in group} == {h}, "bundle %d mixes handlers" % k
        for s in group:
            j = int(s[4])
            assert int(s[0]) >> 8 == j
            assert not seen[j]
            seen[j] = True
            bundle_of[j] = k
    assert seen[4:].all()
    users, rec = {}, {}
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


def test_wide_schedule_length_csg256():
    """The csg256 tape (4693 instructions, dependency depth 31) packs into
    a few dozen single-handler bundles of up to 256 slots."""
    _, bundles, _ = wide(CASES["csg256"]())
    assert len(bundles) <= 80
