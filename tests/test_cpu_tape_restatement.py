"""A second, independent restatement of compute.wgsl's whole-tape passes, in
numpy float32 over many boxes at once, against the oracle's box evaluation:
the forward loop (3632-3774: op_top dispatch, literal-right and literal-left
forms, CONST, RET, `fix` after every instruction) and the reverse AD loop
(3776-3970: output seeded with 1, instructions from the last down to 4, the
zero-sensitivity skip keyed on the operands' use counts, fix(rule) times the
instruction's sensitivity plus the operand's, the larg == rarg case keeping
the second write).  The scene moves its primitives linearly in t, so every
operation of its tape is restated here (the per-op rules are those of
test_cpu_interval_restatement.py, checked there one instruction at a time).
The reference's own four scene tapes run through the same restated passes,
with their elementary functions (sin, cos, exp, pow, floor, mod, atan2)
taken from the oracle one instruction at a time.  Field and all four
argument sensitivities, bit for bit.  No device needed."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from temporalsetinversion_b200 import api
from temporalsetinversion_b200.scenes import IRBuilder
from test_cpu_interval_restatement import _abs_rr, _div_rr_b, _minmax_rr, _sqrt_rr, contains_zero, fix, mul4

f32 = np.float32
ADD, SUB, MUL, DIV, SQR, SQRT, NEG, MIN, MAX, ABS, RET = 5, 6, 7, 8, 11, 12, 16, 17, 18, 19, 28


def linear_scene(seed: int, n: int = 10) -> str:
    """Spheres and boxes moving linearly in t, under min/max, with a
    literal-left subtraction and division and a division by an interval."""
    rng = np.random.default_rng(seed)
    b = IRBuilder()
    X, Y, Z, T = b.X, b.Y, b.Z, b.T
    prims = []
    for i in range(n):
        c = rng.uniform(-0.7, 0.7, 3)
        v = rng.uniform(-0.5, 0.5, 3)
        px = b.sub(X, b.add(b.mul(T, float(v[0])), float(c[0])))
        py = b.sub(Y, b.add(b.mul(T, float(v[1])), float(c[1])))
        pz = b.sub(b.sub(float(c[2]), Z), b.mul(T, float(v[2])))  # c - z (literal-left) - v t
        if i % 2 == 0:
            r = float(rng.uniform(0.1, 0.3))
            d = b.sub(b.sqrt(b.add(b.add(b.mul(px, px), b.mul(py, py)), b.mul(pz, pz))), r)
        else:
            h = rng.uniform(0.05, 0.2, 3)
            d = b.max(b.max(b.sub(b.abs(px), float(h[0])), b.sub(b.abs(py), float(h[1]))),
                      b.sub(b.abs(pz), float(h[2])))
        prims.append(d)
    acc = prims[0]
    for i, d in enumerate(prims[1:]):
        acc = b.max(acc, b.neg(d)) if i % 4 == 3 else b.min(acc, d)
    scale = b.div(1.5, b.add(T, 1.0))               # literal-left division: 1.5 / (t + 1)
    acc = b.div(b.mul(acc, scale), b.add(b.mul(T, 0.25), 1.0))  # a division by an interval
    acc = b.min(acc, b.sub(b.mul(b.neg(Y), -0.5), -0.9))  # a floor plane 0.5 y + 0.9, negative literal product
    return b.text(acc)


def _unpack(w):
    return (int(w) >> 16) & 0xFFFF, int(w) & 0xFFFF


def _forward(op, top, a, b, lit):
    (a0, a1), (b0, b1) = a, b
    L = (f32(lit), f32(lit))
    if top == 1:
        if op == SQR:
            x, y = a0 * a0, a1 * a1
            return np.where(contains_zero(a0, a1), f32(0), np.fmin(x, y)), np.fmax(x, y)
        if op == SQRT:
            return np.sqrt(np.fmax(a0, f32(0))), np.sqrt(np.fmax(a1, f32(0)))
        if op == NEG:
            return -a1, -a0
        if op == ABS:
            cz = contains_zero(a0, a1)
            return (np.where(cz, f32(0), np.where(a1 < 0, -a1, a0)),
                    np.where(cz, np.fmax(-a0, a1), np.where(a1 < 0, -a0, a1)))
        if op == ADD:
            return a0 + L[0], a1 + L[0]
        if op == SUB:
            return a0 - L[0], a1 - L[0]
        if op == MUL:
            return (a0 * L[0], a1 * L[0]) if L[0] >= 0 else (a1 * L[0], a0 * L[0])
        if op == DIV:
            return mul4(a0, a1, L[0], L[1], np.divide)
        if op == MIN:
            return np.fmin(a0, L[0]), np.fmin(a1, L[0])
        if op == MAX:
            return np.fmax(a0, L[0]), np.fmax(a1, L[0])
        if op == RET:
            return a0, a1
    elif top == 0:
        if op == ADD:
            return a0 + b0, a1 + b1
        if op == SUB:
            return a0 - b1, a1 - b0
        if op == MUL:
            return mul4(a0, a1, b0, b1, np.multiply)
        if op == DIV:
            return mul4(a0, a1, b0, b1, np.divide)
        if op == MIN:
            return np.fmin(a0, b0), np.fmin(a1, b1)
        if op == MAX:
            return np.fmax(a0, b0), np.fmax(a1, b1)
        if op == 0:
            return np.full_like(a0, L[0]), np.full_like(a0, L[0])
    elif top == 2:
        if op == SUB:
            return L[0] - b1, L[0] - b0
        if op == DIV:
            return mul4(L[0], L[1], b0, b1, np.divide)
    raise AssertionError("op %d op_top %d is not in the restated set" % (op, top))


def _ones(a, v):
    return np.full_like(a[0], f32(v)), np.full_like(a[0], f32(v))


def _rules(op, top, a, b, lit):
    """The reverse rule(s) of compute.wgsl:2806-2918 as the reverse loop
    calls them: (rule for larg, rule for rarg) by op_top."""
    L = (f32(lit), f32(lit))
    if top == 1:  # RR(larg, I_FROM(literal))[0] or the unary rule
        a0, a1 = a
        r = {SQR: lambda: (a0 * f32(2), a1 * f32(2)), SQRT: lambda: _sqrt_rr(a0, a1, None, None),
             NEG: lambda: _ones(a, -1), ABS: lambda: _abs_rr(a0, a1, None, None),
             ADD: lambda: _ones(a, 1), SUB: lambda: _ones(a, 1),
             MUL: lambda: (np.full_like(a0, L[0]), np.full_like(a0, L[1])),
             DIV: lambda: mul4(f32(1), f32(1), np.full_like(a0, L[0]), np.full_like(a0, L[1]), np.divide),
             MIN: lambda: _minmax_rr(True, True)(a0, a1, L[0], L[1]),
             MAX: lambda: _minmax_rr(False, True)(a0, a1, L[0], L[1]),
             RET: lambda: _ones(a, 1)}[op]()
        return r, None
    if top == 0:
        (a0, a1), (b0, b1) = a, b
        if op == 0:
            return _ones(a, 0), _ones(a, 0)
        return {ADD: lambda: (_ones(a, 1), _ones(a, 1)), SUB: lambda: (_ones(a, 1), _ones(a, -1)),
                MUL: lambda: ((b0, b1), (a0, a1)),
                DIV: lambda: (mul4(f32(1), f32(1), b0, b1, np.divide), _div_rr_b(a0, a1, b0, b1)),
                MIN: lambda: (_minmax_rr(True, True)(a0, a1, b0, b1), _minmax_rr(True, False)(a0, a1, b0, b1)),
                MAX: lambda: (_minmax_rr(False, True)(a0, a1, b0, b1), _minmax_rr(False, False)(a0, a1, b0, b1)),
                }[op]()
    b0, b1 = b  # op_top 2: RR(I_FROM(literal), rarg)[1]
    if op == SUB:
        return None, _ones(b, -1)
    return None, _div_rr_b(np.full_like(b0, L[0]), np.full_like(b0, L[1]), b0, b1)


def restate(tape: np.ndarray, boxes: np.ndarray, forward=None, rules=None) -> np.ndarray:
    """Field interval and the four arguments' sensitivities per box, as the
    oracle's eval_boxes(reverse=True) lays them out."""
    forward = forward or _forward
    rules = rules or _rules
    n = len(tape)
    val = [None] * n
    for q in range(4):
        val[q] = (boxes[:, 2 * q].astype(f32), boxes[:, 2 * q + 1].astype(f32))
    zero = (np.zeros(len(boxes), f32), np.zeros(len(boxes), f32))
    ops = []
    with np.errstate(all="ignore"):
        for j in range(4, n):
            hi, _ = _unpack(tape[j]["opcode_uses"])
            op, top = hi & 0x3FFF, hi >> 14
            la, ra = _unpack(tape[j]["larg_rarg"])
            lit = tape[j]["literal"]
            a = val[la] if top in (0, 1) else zero
            b = val[ra] if top in (0, 2) else zero
            lo_, hi_ = forward(op, top, a, b, lit)
            val[j] = fix(np.asarray(lo_, f32), np.asarray(hi_, f32))
            ops.append((j, op, top, la, ra, lit))
        uses = [_unpack(tape[j]["opcode_uses"])[1] for j in range(n)]
        sens = [zero] * n
        sens[n - 1] = (np.ones(len(boxes), f32), np.ones(len(boxes), f32))
        for j, op, top, la, ra, lit in reversed(ops):
            sj = sens[j]
            zero_j = (sj[0] == 0) & (sj[1] == 0)
            if top == 1:
                skip = zero_j & (uses[la] == 1)
            elif top == 0:
                skip = zero_j & (uses[la] == 1) & (uses[ra] == 1)
            else:
                skip = zero_j & (uses[ra] == 1)
            r_l, r_r = rules(op, top, val[la], val[ra], lit)
            new = {}
            for slot, rule in ((la, r_l), (ra, r_r)):
                if rule is None:
                    continue
                s0, s1 = fix(np.asarray(rule[0], f32), np.asarray(rule[1], f32))
                s0, s1 = mul4(np.broadcast_to(s0, sj[0].shape), np.broadcast_to(s1, sj[0].shape), sj[0], sj[1],
                              np.multiply)
                s0, s1 = s0 + sens[slot][0], s1 + sens[slot][1]
                new[slot] = (np.where(skip, f32(0), s0).astype(f32), np.where(skip, f32(0), s1).astype(f32))
            for slot in ([la] if r_l is not None else []) + ([ra] if r_r is not None else []):
                sens[slot] = new[slot]  # larg first, then rarg: the second write wins when they coincide
    out = np.zeros((len(boxes), 10), f32)
    out[:, 0], out[:, 1] = val[n - 1]
    for q in range(4):
        out[:, 2 + 2 * q], out[:, 3 + 2 * q] = sens[q]
    return out


def _boxes(rng, n):
    lo = rng.uniform(-1.2, 1.2, (n, 3)).astype(f32)
    w = (f32(10.0) * np.exp2(-rng.integers(2, 9, n))).astype(f32)
    t0 = rng.uniform(0, 1, n).astype(f32)
    dt = np.where(rng.uniform(size=n) < 0.25, f32(0), rng.uniform(0, 0.05, n).astype(f32)).astype(f32)
    b = np.zeros((n, 8), f32)
    for a in range(3):
        b[:, 2 * a], b[:, 2 * a + 1] = lo[:, a], (lo[:, a] + w).astype(f32)
    b[:, 6], b[:, 7] = t0, (t0 + dt).astype(f32)
    return b


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_whole_tape_matches_restatement(seed):
    oracle.build()
    tape = api.IR.new(linear_scene(seed)).gpu_instructions
    ops = {((int(w) >> 16) & 0x3FFF, int(w) >> 30) for w in tape["opcode_uses"][4:]}
    assert {(DIV, 2), (SUB, 2), (DIV, 0), (MIN, 0), (MAX, 0), (SQRT, 1), (ABS, 1), (NEG, 1)} <= ops, ops
    rng = np.random.default_rng(seed)
    boxes = _boxes(rng, 3000)
    got = oracle.eval_boxes(tape, boxes, reverse=True).astype(f32)
    want = restate(tape, boxes)
    bad = np.nonzero(np.any(got.view(np.uint32) != want.view(np.uint32), axis=1))[0]
    assert len(bad) == 0, "%d of %d boxes differ, e.g. box %s: oracle %s restated %s" % (
        len(bad), len(boxes), boxes[bad[0]], got[bad[0]], want[bad[0]])
    # the boxes reach both sides of the surface and zero sensitivities (the skip rule)
    assert (got[:, 0] > 0).any() and (got[:, 1] < 0).any()


# Elementary functions (SIN 14, COS 15, EXP 9, LOG 10, POW 13, FLOOR 25,
# MOD 29, ATAN2 30) are the driver's in the reference and the library's own
# fixed sequences here; for the reference's scene tapes their value and rule
# are taken from the oracle one instruction at a time, everything else (the
# sequencing and every other operation) is restated above.
ELEMENTARY = {9, 10, 13, 14, 15, 25, 29, 30}


def _one_op_tape(op, top, lit):
    from temporalsetinversion_b200.api import GPU_INSTR_DTYPE
    t = np.zeros(5, GPU_INSTR_DTYPE)
    for q in range(4):
        t[q]["index_"] = q
        t[q]["opcode_uses"] = (((q + 1) | (3 << 14)) << 16) | (1 if q < 2 else 0)
    t[4]["index_"] = 4
    t[4]["opcode_uses"] = ((op | (top << 14)) << 16) | 1
    t[4]["larg_rarg"] = (0 << 16) | (1 if top == 0 else 0)
    t[4]["literal"] = lit
    return t


def _oracle_op(op, top, a, b, lit):
    """(value, rule for larg, rule for rarg) of one elementary instruction."""
    boxes = np.zeros((len(a[0]), 8), f32)
    boxes[:, 0], boxes[:, 1] = a
    if top == 0:
        boxes[:, 2], boxes[:, 3] = b
    boxes[:, 6:8] = (0.0, 1.0)  # a time interval: the reverse pass runs
    out = oracle.eval_boxes(_one_op_tape(op, top, lit), boxes, reverse=True).astype(f32)
    return (out[:, 0], out[:, 1]), (out[:, 2], out[:, 3]), ((out[:, 4], out[:, 5]) if top == 0 else None)


def restate_with_elementary(tape: np.ndarray, boxes: np.ndarray) -> np.ndarray:
    """restate() for tapes that also hold elementary functions."""
    cache = {}

    def fwd(op, top, a, b, lit):
        if op in ELEMENTARY and top in (0, 1):
            key = (op, top, id(a), id(b), float(lit))
            cache[key] = _oracle_op(op, top, a, b, lit)
            return cache[key][0]
        return _forward(op, top, a, b, lit)

    def rules(op, top, a, b, lit):
        if op in ELEMENTARY and top in (0, 1):
            _, r_l, r_r = cache.get((op, top, id(a), id(b), float(lit))) or _oracle_op(op, top, a, b, lit)
            return r_l, r_r
        return _rules(op, top, a, b, lit)

    return restate(tape, boxes, fwd, rules)


@pytest.mark.parametrize("scene", ["cables", "cradle", "piano", "sponza"])
def test_reference_scene_tapes_match_restatement(scene):
    """The reference's own scene tapes (scenes/*.ll, lowered as committed
    under tests/golden/tapes): field and argument sensitivities bit for bit
    on random space-time boxes."""
    from golden.make_golden import load_tape
    oracle.build()
    tape = load_tape(scene)
    rng = np.random.default_rng(sum(map(ord, scene)))
    boxes = _boxes(rng, 2000)
    boxes[:, 0:6] = (boxes[:, 0:6] * f32(4)).astype(f32)  # the scenes span the [-5, 5] root box
    got = oracle.eval_boxes(tape, boxes, reverse=True).astype(f32)
    want = restate_with_elementary(tape, boxes)
    bad = np.nonzero(np.any(got.view(np.uint32) != want.view(np.uint32), axis=1))[0]
    assert len(bad) == 0, "%d of %d boxes differ, e.g. box %s: oracle %s restated %s" % (
        len(bad), len(boxes), boxes[bad[0]], got[bad[0]], want[bad[0]])
    assert ((got[:, 0] <= 0) & (got[:, 1] >= 0)).sum() > 20
