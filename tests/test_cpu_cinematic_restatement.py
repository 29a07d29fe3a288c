"""The oracle's cinematic pieces against separately written restatements:
the PCG random numbers of frand / frand0to1 (compute.wgsl:2451-2472) bit
for bit from Python integers, the sky model (sunsky 520-677) against a
float64 evaluation of the same formulas, the sRGB curve (4600-4607), and
the oracle's cos / acos against float64 within a few ulp."""
from __future__ import annotations

import math

import numpy as np

import oracle


def _pcg_word(s: int) -> int:
    w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & 0xFFFFFFFF
    return ((w >> 22) ^ w) & 0xFFFFFFFF


def test_frand_sequence_bit_exact():
    for seed in (0, 1, 12345, 0xDEADBEEF, 4294967295):
        got = oracle.frand_seq(seed, 64)
        s = seed
        want = []
        for i in range(64):
            s = (s * 747796405 + 1) & 0xFFFFFFFF
            x = np.float32(_pcg_word(s)) / np.float32(4294967295.0)
            want.append(np.float32(np.float32(x * np.float32(2.0)) - np.float32(1.0)) if i % 2 == 0 else x)
        assert np.array_equal(got, np.asarray(want, np.float32)), seed


def _sky64(view, sun):
    """sunsky (compute.wgsl:520-677) in float64: turbidity 1, sunSize 1,
    sun intensity 1000; returns 0.01 * sky."""
    pi = math.pi
    px, py = (sun[0] - 0.0) * 6.28, (sun[1] - 0.5) * 3.14
    sd = np.array([math.cos(px) * math.sin(py), math.sin(px) * math.sin(py), math.cos(py)])
    sd = sd / np.linalg.norm(sd)
    v = np.asarray(view, np.float64)
    cvs, csu, cuv = float(v @ sd), float(sd[2]), float(v[2])
    sunE = 1000.0 * max(0.0, 1.0 - math.exp(-((1.6110731611233942 - math.acos(csu)) / 1.5)))
    ray = np.array([5.176821105123963e-6, 1.2785348189936485e-5, 2.8530756026157178e-5])
    lam = np.array([6.8e-7, 5.5e-7, 4.5e-7])
    K = np.array([0.686, 0.678, 0.666])
    c = 0.2 * 1.0 * 1e-17
    mie = 0.434 * c * pi * (2.0 * pi / lam) ** 2 * K * 0.005
    zen = max(0.0, cuv)
    with np.errstate(divide="ignore"):
        fex = np.exp(-(ray * (8400.0 / zen) + mie * (1250.0 / zen)))
    rphase = 3.0 / (16.0 * pi) * (1.0 + cvs ** 2)
    g = 0.8
    hg = 1.0 / (4.0 * pi) * ((1.0 - g ** 2) / ((1.0 - 2.0 * g * cvs) + g ** 2) ** 1.5)
    se = sunE * ((ray * rphase + mie * hg) / (ray + mie))
    sky = se * (1.0 - fex)
    t = min(max((1.0 - sd[2]) ** 5, 0.0), 1.0)
    sky = sky * ((1.0 - t) + np.sqrt(se * fex) * t)
    return 0.01 * sky


def test_sky_matches_float64_formula():
    rng = np.random.default_rng(3)
    for sun in ((-0.1, 0.7), (0.36, 0.72), (0.63, 0.65)):
        for _ in range(200):
            v = rng.normal(size=3)
            v[2] = abs(v[2]) + 0.05  # above the horizon
            v = v / np.linalg.norm(v)
            got = oracle.sunsky(v.astype(np.float32), sun).astype(np.float64)
            want = _sky64(v.astype(np.float32).astype(np.float64), sun)
            assert np.all(np.isfinite(got))
            assert np.allclose(got, want, rtol=2e-4, atol=1e-7), (sun, v, got, want)


def test_srgb_curve():
    lib = oracle.load()
    for x in (-1.0, 0.0, 0.001, 0.0031308, 0.004, 0.2, 0.5, 1.0, 2.0):
        got = lib.oracle_linear_to_srgb(x)
        r = min(max(x, 0.0), 1.0)
        want = r * 12.92 if r < 0.0031308 else 1.055 * r ** (1.0 / 2.4) - 0.055
        assert abs(got - want) <= 2e-6 + 1e-5 * abs(want), (x, got, want)


def test_cos_acos_accuracy():
    lib = oracle.load()
    xs = np.linspace(-40.0, 40.0, 4001).astype(np.float32)
    got = np.array([lib.oracle_cos(float(x)) for x in xs], np.float64)
    assert np.max(np.abs(got - np.cos(xs.astype(np.float64)))) < 4e-7
    ys = np.linspace(-1.0, 1.0, 2001).astype(np.float32)
    got = np.array([lib.oracle_acos(float(y)) for y in ys], np.float64)
    assert np.max(np.abs(got - np.arccos(ys.astype(np.float64)))) < 2e-6
