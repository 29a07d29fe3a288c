"""A second, independent restatement of compute.wgsl's interval operations
(2539-2637, 2689-2698), their reverse rules as the reverse pass applies them
(2806-2918, 3776-3955) and `fix` (3462-3472), written here in numpy float32,
against the oracle's evaluation of one-instruction tapes: bit for bit on
random intervals, including divisors and radicands that contain zero.  The
device kernels equal the oracle (tests/test_gpu_ops.py), so this pins both
to the reference's formulas for these operations.  No device needed."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from temporalsetinversion_b200 import api
from temporalsetinversion_b200.scenes import IRBuilder

f32 = np.float32
BIG = f32(1000000.0)  # compute.wgsl:2534-2536


def fix(lo, hi):
    lo = np.where(np.isnan(lo), -BIG, lo).astype(f32)
    hi = np.where(np.isnan(hi), BIG, hi).astype(f32)
    return np.fmax(lo, -BIG), np.fmin(hi, BIG)


def contains_zero(lo, hi):
    return (lo <= 0) & (0 <= hi)


def mul4(alo, ahi, blo, bhi, op):
    x, y, z, w = op(alo, blo), op(alo, bhi), op(ahi, blo), op(ahi, bhi)
    return np.fmin(np.fmin(x, y), np.fmin(z, w)), np.fmax(np.fmax(x, y), np.fmax(z, w))


C = f32(0.75)
CN = f32(-1.5)

# name -> (IR builder of the op on x and y, restatement on (alo, ahi, blo, bhi))
OPS = {
    "ADD_II": (lambda b: b.add(b.X, b.Y), lambda a0, a1, b0, b1: (a0 + b0, a1 + b1)),
    "ADD_IF": (lambda b: b.add(b.X, float(C)), lambda a0, a1, b0, b1: (a0 + C, a1 + C)),
    "SUB_II": (lambda b: b.sub(b.X, b.Y), lambda a0, a1, b0, b1: (a0 - b1, a1 - b0)),
    "SUB_IF": (lambda b: b.sub(b.X, float(C)), lambda a0, a1, b0, b1: (a0 - C, a1 - C)),
    "SUB_FI": (lambda b: b.sub(float(C), b.X), lambda a0, a1, b0, b1: (C - a1, C - a0)),
    "MUL_II": (lambda b: b.mul(b.X, b.Y), lambda a0, a1, b0, b1: mul4(a0, a1, b0, b1, np.multiply)),
    "MUL_IF+": (lambda b: b.mul(b.X, float(C)), lambda a0, a1, b0, b1: (a0 * C, a1 * C)),
    "MUL_IF-": (lambda b: b.mul(b.X, float(CN)), lambda a0, a1, b0, b1: (a1 * CN, a0 * CN)),
    "DIV_II": (lambda b: b.div(b.X, b.Y), lambda a0, a1, b0, b1: mul4(a0, a1, b0, b1, np.divide)),
    "DIV_IF": (lambda b: b.div(b.X, float(CN)), lambda a0, a1, b0, b1: mul4(a0, a1, CN, CN, np.divide)),
    "SQR": (lambda b: b.mul(b.X, b.X),
            lambda a0, a1, b0, b1: (np.where(contains_zero(a0, a1), f32(0), np.fmin(a0 * a0, a1 * a1)),
                                    np.fmax(a0 * a0, a1 * a1))),
    "SQRT": (lambda b: b.sqrt(b.X),
             lambda a0, a1, b0, b1: (np.sqrt(np.fmax(a0, f32(0))), np.sqrt(np.fmax(a1, f32(0))))),
    "NEG": (lambda b: b.neg(b.X), lambda a0, a1, b0, b1: (-a1, -a0)),
    "ABS": (lambda b: b.abs(b.X),
            lambda a0, a1, b0, b1: (np.where(contains_zero(a0, a1), f32(0), np.where(a1 < 0, -a1, a0)),
                                    np.where(contains_zero(a0, a1), np.fmax(-a0, a1), np.where(a1 < 0, -a0, a1)))),
    "MIN_II": (lambda b: b.min(b.X, b.Y), lambda a0, a1, b0, b1: (np.fmin(a0, b0), np.fmin(a1, b1))),
    "MAX_II": (lambda b: b.max(b.X, b.Y), lambda a0, a1, b0, b1: (np.fmax(a0, b0), np.fmax(a1, b1))),
    "MIN_IF": (lambda b: b.min(b.X, float(C)), lambda a0, a1, b0, b1: (np.fmin(a0, C), np.fmin(a1, C))),
    "MAX_IF": (lambda b: b.max(b.X, float(C)), lambda a0, a1, b0, b1: (np.fmax(a0, C), np.fmax(a1, C))),
}


def _intervals(rng, n):
    a = rng.uniform(-3, 3, (n, 2)).astype(f32)
    a.sort(axis=1)
    # some zero-width and huge intervals, and bounds at exactly 0
    a[: n // 16] = a[: n // 16, :1]
    a[n // 16: n // 8] *= f32(1e7)
    a[n // 8: n // 8 + 4] = np.array([[0, 1], [-1, 0], [0, 0], [-2, -1]], f32)
    return a


@pytest.mark.parametrize("name", sorted(OPS))
def test_interval_op_matches_restatement(name):
    oracle.build()
    build, ref = OPS[name]
    b = IRBuilder()
    tape = api.IR.new(b.text(build(b))).gpu_instructions
    rng = np.random.default_rng(sum(map(ord, name)))
    n = 4096
    x, y = _intervals(rng, n), _intervals(rng, n)[rng.permutation(n)]
    boxes = np.zeros((n, 8), f32)
    boxes[:, 0:2], boxes[:, 2:4] = x, y
    got = oracle.eval_boxes(tape, boxes, reverse=False)[:, 0:2]
    with np.errstate(all="ignore"):
        lo, hi = ref(x[:, 0], x[:, 1], y[:, 0], y[:, 1])
        lo, hi = fix(np.asarray(lo, f32), np.asarray(hi, f32))
    want = np.stack([lo, hi], axis=1).astype(f32)
    bad = np.nonzero(got.view(np.uint32) != want.view(np.uint32))[0]
    assert len(bad) == 0, "%s: %d of %d differ, e.g. x=%s y=%s got %s want %s" % (
        name, len(bad), n, x[bad[0]], y[bad[0]], got[bad[0]], want[bad[0]])


# reverse rules (compute.wgsl:2806-2918, 2638-2646) as the reverse pass
# applies them to the operands of a one-instruction tape whose output has
# sensitivity [1, 1] (3866-3874, 3918-3930, 3952-3955): fix(rule), times the
# output's sensitivity, plus the operand's sensitivity so far ([0, 0])
ONE = (f32(1), f32(1))


def _const(c):
    return lambda a0, a1, b0, b1: (np.full_like(a0, f32(c)), np.full_like(a0, f32(c)))


def _minmax_rr(is_min, first):
    def rr(a0, a1, b0, b1):
        a_below, b_below = a1 < b0, b1 < a0
        if is_min:
            la = np.where(a_below, 1, np.where(b_below, 0, 1))
            lb = np.where(a_below, 0, np.where(b_below, 1, 1))
        else:
            la = np.where(a_below, 0, np.where(b_below, 1, 1))
            lb = np.where(a_below, 1, np.where(b_below, 0, 1))
        v = (la if first else lb).astype(f32)
        return v, v
    return rr


def _div_rr_b(a0, a1, b0, b1):
    s0 = np.where(contains_zero(b0, b1), f32(0), np.fmin(b0 * b0, b1 * b1))
    s1 = np.fmax(b0 * b0, b1 * b1)
    q0, q1 = mul4(a0, a1, s0, s1, np.divide)
    return -q1, -q0


def _sqrt_rr(a0, a1, b0, b1):
    s0, s1 = np.sqrt(np.fmax(a0, f32(0))), np.sqrt(np.fmax(a1, f32(0)))
    lo, hi = mul4(f32(1), f32(1), s0 * f32(2), s1 * f32(2), np.divide)
    return lo, np.fmin(hi, BIG)


def _abs_rr(a0, a1, b0, b1):
    cz = contains_zero(a0, a1)
    return (np.where(cz, f32(-1), np.where(a1 < 0, f32(-1), f32(1))),
            np.where(cz, f32(1), np.where(a1 < 0, f32(-1), f32(1))))


REV = {  # name -> (rule for x, rule for y or None)
    "ADD_II": (_const(1), _const(1)),
    "ADD_IF": (_const(1), None),
    "SUB_II": (_const(1), _const(-1)),
    "SUB_IF": (_const(1), None),
    "SUB_FI": (_const(-1), None),
    "MUL_II": (lambda a0, a1, b0, b1: (b0, b1), lambda a0, a1, b0, b1: (a0, a1)),
    "MUL_IF+": (_const(C), None),
    "MUL_IF-": (_const(CN), None),
    "DIV_II": (lambda a0, a1, b0, b1: mul4(f32(1), f32(1), b0, b1, np.divide), _div_rr_b),
    "DIV_IF": (_const(f32(1) / CN), None),
    "SQR": (lambda a0, a1, b0, b1: (a0 * f32(2), a1 * f32(2)), None),
    "SQRT": (_sqrt_rr, None),
    "NEG": (_const(-1), None),
    "ABS": (_abs_rr, None),
    "MIN_II": (_minmax_rr(True, True), _minmax_rr(True, False)),
    "MAX_II": (_minmax_rr(False, True), _minmax_rr(False, False)),
    "MIN_IF": (lambda a0, a1, b0, b1: _minmax_rr(True, True)(a0, a1, C, C), None),
    "MAX_IF": (lambda a0, a1, b0, b1: _minmax_rr(False, True)(a0, a1, C, C), None),
}


def _apply(rule, x, y):
    lo, hi = rule(x[:, 0], x[:, 1], y[:, 0], y[:, 1])
    lo, hi = fix(np.asarray(lo, f32), np.asarray(hi, f32))
    lo, hi = mul4(lo, hi, ONE[0], ONE[1], np.multiply)
    return np.stack([lo + f32(0), hi + f32(0)], axis=1).astype(f32)


@pytest.mark.parametrize("name", sorted(REV))
def test_reverse_rule_matches_restatement(name):
    oracle.build()
    build, _ = OPS[name]
    rule_x, rule_y = REV[name]
    b = IRBuilder()
    tape = api.IR.new(b.text(build(b))).gpu_instructions
    rng = np.random.default_rng(7 + sum(map(ord, name)))
    n = 4096
    x, y = _intervals(rng, n), _intervals(rng, n)[rng.permutation(n)]
    boxes = np.zeros((n, 8), f32)
    boxes[:, 0:2], boxes[:, 2:4] = x, y
    boxes[:, 6:8] = np.array([0.0, 1.0], f32)  # a time interval: the reverse pass runs
    out = oracle.eval_boxes(tape, boxes, reverse=True)
    with np.errstate(all="ignore"):
        checks = [("x", out[:, 2:4], _apply(rule_x, x, y))]
        if rule_y is not None:
            checks.append(("y", out[:, 4:6], _apply(rule_y, x, y)))
    for arg, got, want in checks:
        bad = np.nonzero(got.astype(f32).view(np.uint32) != want.view(np.uint32))[0]
        assert len(bad) == 0, "%s d/d%s: %d of %d differ, e.g. x=%s y=%s got %s want %s" % (
            name, arg, len(bad), n, x[bad[0]], y[bad[0]], got[bad[0]], want[bad[0]])
