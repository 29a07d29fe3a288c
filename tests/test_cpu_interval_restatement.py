"""A second, independent restatement of compute.wgsl's interval operations
(2539-2637, 2689-2698) and `fix` (3462-3472), written here in numpy float32,
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
