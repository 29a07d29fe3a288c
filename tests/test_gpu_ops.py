"""Interval instructions and f32 math on the GPU against the CPU oracle.

Round-to-nearest mode must agree bit for bit (forward value and the reverse
sensitivities of x, y, z, t) for every opcode and operand kind the lowering
produces, including the reference's quirks (literal-left ops other than
SUB/DIV give -inf, MOD has no op_top-0 reverse rule, ATAN2 swaps its
operands).  Directed mode must enclose dense FP64 point samples."""
from __future__ import annotations

import math
import zlib

import numpy as np
import pytest

import oracle
from temporalsetinversion_b200 import Tape, api

HDR = "define dso_local float @_Z1fffff(float %0, float %1, float %2, float %3) local_unnamed_addr #5 {\n"


def ll(*lines):
    return HDR + "\n".join("  " + s for s in lines) + "\n}\n"


# one scene per opcode / operand kind; %0..%3 are x, y, z, t
OPS = {
    "add_ii": ll("%5 = fadd float %0, %1", "ret float %5"),
    "add_if": ll("%5 = fadd float %0, 0x3FF8000000000000", "ret float %5"),
    "add_fi_bad": ll("%5 = fadd float 0x3FF8000000000000, %0", "ret float %5"),
    "sub_ii": ll("%5 = fsub float %0, %1", "ret float %5"),
    "sub_fi": ll("%5 = fsub float 0x3FF8000000000000, %1", "ret float %5"),
    "mul_ii": ll("%5 = fmul float %0, %1", "ret float %5"),
    "mul_if_neg": ll("%5 = fmul float %0, 0xC004000000000000", "ret float %5"),
    "sqr": ll("%5 = fmul float %0, %0", "ret float %5"),
    "div_ii": ll("%5 = fdiv float %0, %1", "ret float %5"),
    "div_fi": ll("%5 = fdiv float 1.000000e+00, %1", "ret float %5"),
    "div_if": ll("%5 = fdiv float %1, 3.000000e+00", "ret float %5"),
    "neg": ll("%5 = fneg float %2", "ret float %5"),
    "sqrt": ll("%5 = tail call float @sqrtf(float %0) #10", "ret float %5"),
    "exp": ll("%5 = tail call float @expf(float %0) #10", "ret float %5"),
    "log": ll("%5 = tail call float @logf(float %0) #10", "ret float %5"),
    "sin": ll("%5 = fmul float %0, 0x4014000000000000", "%6 = tail call float @sinf(float %5) #10", "ret float %6"),
    "cos": ll("%5 = fmul float %3, 0x4024000000000000", "%6 = tail call float @cosf(float %5) #10", "ret float %6"),
    "abs": ll("%5 = tail call float @llvm.fabs.f32(float %1) #10", "ret float %5"),
    "floor": ll("%5 = fmul float %0, 3.000000e+00", "%6 = tail call float @llvm.floor.f32(float %5) #10",
                "ret float %6"),
    "min_ii": ll("%5 = tail call float @llvm.minnum.f32(float %0, float %1) #10", "ret float %5"),
    "max_ii": ll("%5 = tail call float @llvm.maxnum.f32(float %0, float %1) #10", "ret float %5"),
    "min_if": ll("%5 = tail call float @llvm.minnum.f32(float %0, float 5.000000e-01) #10", "ret float %5"),
    "max_if": ll("%5 = tail call float @llvm.maxnum.f32(float %0, float -5.000000e-01) #10", "ret float %5"),
    "pow_if": ll("%5 = tail call float @powf(float %0, float 3.000000e+00) #10", "ret float %5"),
    "pow_ii": ll("%5 = tail call float @powf(float %0, float %3) #10", "ret float %5"),
    "mod_if": ll("%5 = tail call float @fmodf(float %0, float 7.500000e-01) #10", "ret float %5"),
    "mod_ii": ll("%5 = tail call float @fmodf(float %0, float %1) #10", "ret float %5"),
    "atan2_ii": ll("%5 = tail call float @atan2f(float %0, float %1) #10", "ret float %5"),
    "atan2_if": ll("%5 = tail call float @atan2f(float %1, float 5.000000e-01) #10", "ret float %5"),
    "shared_operand": ll("%5 = fadd float %0, %0", "%6 = fmul float %5, %1", "%7 = fsub float %6, %5",
                         "ret float %7"),
    "chain": ll("%5 = fmul float %0, %0", "%6 = fmul float %1, %1", "%7 = fadd float %5, %6",
                "%8 = tail call float @sqrtf(float %7) #10", "%9 = fadd float %8, -5.000000e-01",
                "%10 = tail call float @llvm.minnum.f32(float %9, float %2) #10", "ret float %10"),
}


def random_boxes(n, rng, scale=2.0):
    lo = rng.uniform(-scale, scale, (n, 4)).astype(np.float32)
    w = (rng.uniform(0, 1, (n, 4)) ** 3 * scale).astype(np.float32)
    w[rng.uniform(size=(n, 4)) < 0.2] = 0.0  # degenerate (point) intervals
    hi = (lo + w).astype(np.float32)
    b = np.empty((n, 8), np.float32)
    b[:, 0::2], b[:, 1::2] = lo, hi
    # intervals starting at an exact zero, and [-0, +0]
    b[: n // 16, 0] = 0.0
    b[: n // 16, 1] = np.abs(b[: n // 16, 1])
    b[n // 16: n // 8, 2:4] = [-0.0, 0.0]
    assert np.all(b[:, 0::2] <= b[:, 1::2])
    return b


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(OPS))
def test_op_rn_bit_exact(device, name):
    tape = api.IR.new(OPS[name]).gpu_instructions
    boxes = random_boxes(4096, np.random.default_rng(zlib.crc32(name.encode())))
    g = Tape.upload(device, tape).eval_boxes(boxes, rounding_mode=0, reverse=True)
    o = oracle.eval_boxes(tape, boxes, reverse=True)
    same = (g == o) | (np.isnan(g) & np.isnan(o))
    bad = np.nonzero(~same.all(axis=1))[0]
    assert len(bad) == 0, "%s: %d boxes differ, first box %s gpu %s oracle %s" % (
        name, len(bad), boxes[bad[0]], g[bad[0]], o[bad[0]])


def _point_f64(name, x, y, z, t):
    """FP64 meaning of each test tape (MOD is floor-mod and ATAN2 takes its
    operands swapped, as the reference's interval ops define them)."""
    m = {
        "add_ii": lambda: x + y, "add_if": lambda: x + 1.5, "sub_ii": lambda: x - y, "sub_fi": lambda: 1.5 - y,
        "mul_ii": lambda: x * y, "mul_if_neg": lambda: x * -2.5, "sqr": lambda: x * x, "div_ii": lambda: x / y,
        "div_fi": lambda: 1.0 / y, "div_if": lambda: y / 3.0, "neg": lambda: -z,
        "sqrt": lambda: np.sqrt(np.maximum(x, 0)), "exp": lambda: np.exp(x), "abs": lambda: np.abs(y),
        "sin": lambda: np.sin(5 * x), "cos": lambda: np.cos(10 * t), "floor": lambda: np.floor(3 * x),
        "min_ii": lambda: np.minimum(x, y), "max_ii": lambda: np.maximum(x, y), "min_if": lambda: np.minimum(x, 0.5),
        "max_if": lambda: np.maximum(x, -0.5), "pow_if": lambda: x ** 3, "mod_if": lambda: x - 0.75 * np.floor(x / 0.75),
        "atan2_ii": lambda: np.arctan2(y, x), "atan2_if": lambda: np.arctan2(0.5, y),
        "chain": lambda: np.minimum(np.sqrt(x * x + y * y) - 0.5, z),
        "shared_operand": lambda: (x + x) * y - (x + x),
    }
    return m[name]() if name in m else None


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["add_ii", "add_if", "sub_ii", "sub_fi", "mul_ii", "mul_if_neg", "sqr", "div_ii",
                                  "div_if", "neg", "sqrt", "exp", "abs", "sin", "cos", "floor", "min_ii", "max_ii",
                                  "min_if", "max_if", "pow_if", "mod_if", "atan2_ii", "atan2_if", "chain",
                                  "shared_operand"])
def test_op_directed_encloses_fp64(device, name):
    rng = np.random.default_rng(7)
    tape = api.IR.new(OPS[name]).gpu_instructions
    boxes = random_boxes(512, rng, scale=2.0)
    g = Tape.upload(device, tape).eval_boxes(boxes, rounding_mode=1, reverse=False)
    s = rng.uniform(0, 1, (512, 64, 4))
    lo, hi = boxes[:, 0::2].astype(np.float64), boxes[:, 1::2].astype(np.float64)
    pts = lo[:, None, :] + s * (hi - lo)[:, None, :]
    pts[:, 0, :], pts[:, 1, :] = lo, hi
    with np.errstate(all="ignore"):
        v = _point_f64(name, pts[..., 0], pts[..., 1], pts[..., 2], pts[..., 3])
    fin = np.isfinite(v)
    below = fin & (v < g[:, 0:1].astype(np.float64))
    above = fin & (v > g[:, 1:2].astype(np.float64))
    assert not below.any() and not above.any(), "%s: sample outside the directed enclosure" % name


@pytest.mark.gpu
def test_math_bit_exact_and_accurate(device):
    rng = np.random.default_rng(3)
    lib = oracle.load()
    n = 1 << 16
    cases = {
        0: (np.concatenate([rng.uniform(-10, 10, n), rng.uniform(-6000, 6000, n // 4), [0.0, -0.0, 1e-30]]), None),
        1: (np.concatenate([rng.uniform(-100, 90, n), [0.0, -0.0, 88.7, -103.9, 89.0, -110.0]]), None),
        2: (np.concatenate([np.exp(rng.uniform(-80, 80, n)), [0.0, 1.0, 2.0, 1e-40, 3e38]]), None),
        3: (rng.uniform(-5, 5, n), rng.uniform(-5, 5, n)),
        4: (rng.uniform(-3, 3, n), rng.integers(-6, 7, n).astype(np.float64)),
    }
    ref_fn = {0: lib.oracle_sin, 1: lib.oracle_exp, 2: lib.oracle_log}
    np_fn = {0: np.sin, 1: np.exp, 2: np.log}
    for which, (a, b) in cases.items():
        a32 = a.astype(np.float32)
        b32 = np.zeros_like(a32) if b is None else b.astype(np.float32)
        g = device.math(which, a32, b32)
        if which in ref_fn:
            o = np.array([ref_fn[which](float(x)) for x in a32], np.float32)
        elif which == 3:
            o = np.array([lib.oracle_atan2(float(x), float(y)) for x, y in zip(a32, b32)], np.float32)
        else:
            o = np.array([lib.oracle_powi(float(x), int(y)) for x, y in zip(a32, b32)], np.float32)
        same = (g == o) | (np.isnan(g) & np.isnan(o))
        assert same.all(), "math %d: gpu and oracle differ" % which
        # accuracy against float64 (ulps of the f32 result), where the
        # reduction is exact (sin) and the result is normal
        if which in np_fn:
            with np.errstate(all="ignore"):
                ref = np_fn[which](a32.astype(np.float64))
            sel = np.isfinite(ref) & (np.abs(ref) > 1e-30) & (np.abs(ref) < 3.0e38) & (np.abs(a32) < 6000)
            if which == 0:
                sel &= np.abs(ref) > 1e-3
            ulp = np.spacing(np.abs(ref[sel]).astype(np.float32)).astype(np.float64)
            err = np.abs(g[sel].astype(np.float64) - ref[sel]) / ulp
            assert err.max() <= 3.0, "math %d: max error %.2f ulp" % (which, err.max())
        if which == 3:
            ref = np.arctan2(a32.astype(np.float64), b32.astype(np.float64))
            ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
            err = np.abs(g.astype(np.float64) - ref) / np.maximum(ulp, 1e-45)
            assert err[np.abs(ref) > 1e-6].max() <= 3.0


@pytest.mark.gpu
def test_min_max_semantics(device):
    a = np.array([-0.0, 0.0, 1.0, np.nan, 2.0, -0.0, np.nan], np.float32)
    b = np.array([0.0, -0.0, np.nan, 1.0, 2.0, -0.0, np.nan], np.float32)
    mn, mx = device.math(5, a, b), device.math(6, a, b)
    assert [np.signbit(v) for v in mn[:2]] == [True, True]
    assert [np.signbit(v) for v in mx[:2]] == [False, False]
    assert mn[2] == 1.0 and mn[3] == 1.0 and mx[2] == 1.0 and mx[3] == 1.0 and np.isnan(mn[6])
    hw_mn, hw_mx = device.math(7, a, b), device.math(8, a, b)  # raw fminf / fmaxf
    lib = oracle.load()
    for i in range(len(a)):
        for which, fn in ((5, lib.oracle_fmin), (6, lib.oracle_fmax), (7, lib.oracle_fmin), (8, lib.oracle_fmax)):
            o = np.float32(fn(float(a[i]), float(b[i])))
            g = {5: mn, 6: mx, 7: hw_mn, 8: hw_mx}[which][i]
            assert (np.isnan(o) and np.isnan(g)) or (o == g and np.signbit(o) == np.signbit(g))
