"""A second, independent restatement of compute.wgsl's per-cell temporal
logic (cell time range 3603-3613, temporal error bound and Lipschitz
correction 3971-3996, fast flag 4003-4009, classification and re-enqueue
4011-4033), in numpy float32, against the oracle's octree: every cell of
two levels that three frames evaluate, with time_err accumulating, cells
re-enqueued and parents turning fast; the point-sampled leaves
(3603-3621); and the swept-volume branch (3603-3605, 3629, 4028-4044).  The cells' field and sensitivities
come from the oracle's box evaluation, itself checked operation by
operation in test_cpu_interval_restatement.py.  No device needed."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from temporalsetinversion_b200 import api, scenes

f32 = np.float32
INF = f32(np.inf)


def abs_i(lo, hi):  # ABS_I, 2628-2636
    if lo <= 0 <= hi:
        return f32(0), max(-lo, hi)
    if hi < 0:
        return -hi, -lo
    return lo, hi


def sqr_i(lo, hi):  # SQR_I, 2689-2697
    x, y = f32(lo * lo), f32(hi * hi)
    if lo <= 0 <= hi:
        return f32(0), max(x, y)
    return min(x, y), max(x, y)


def mul_if(lo, hi, b):  # MUL_IF, 2559-2565
    return (f32(lo * b), f32(hi * b)) if b >= 0 else (f32(hi * b), f32(lo * b))


def cell_update(F, sens, t0, t1, delta, time_err_old, children, lipschitz):
    """time_err, fast, f, enqueued of a non-new cell evaluated over [t0, t1]."""
    df_dt = sens[3]
    dt = f32(f32(t1) - f32(t0))
    df = mul_if(df_dt[0], df_dt[1], dt)
    W = mul_if(f32(-1), f32(1), f32(F[1] - F[0]))
    if df[1] < W[0] or W[1] < df[0]:  # CAP_II, 2664-2670
        df = (INF, -INF)
    else:
        df = (max(df[0], W[0]), min(df[1], W[1]))
    if lipschitz and abs_i(*df)[1] != 0:
        s = [sqr_i(*sens[q]) for q in range(3)]
        acc = (f32(s[1][0] + s[2][0]), f32(s[1][1] + s[2][1]))
        acc = (f32(s[0][0] + acc[0]), f32(s[0][1] + acc[1]))
        root = (np.sqrt(max(acc[0], f32(0))), np.sqrt(max(acc[1], f32(0))))
        lb = abs_i(*root)[0]
        if not np.isnan(lb):
            q = [f32(df[0] / lb), f32(df[1] / lb)]  # DIV_IF = DIV_II with [lb, lb]
            df = (min(q), max(q))
    if df[0] == -INF or df[1] == INF or np.isnan(df[0]) or np.isnan(df[1]):
        df = (f32(delta), f32(delta))
    time_err = f32(time_err_old + np.clip(abs_i(*df)[1], f32(0), f32(delta)))
    fast = f32(1) if abs_i(*df)[1] >= f32(delta) else f32(0)
    enq = False
    if F[0] <= 0 <= F[1]:
        f = f32(0)
        bad_dt = np.isnan(df_dt[0]) or np.isnan(df_dt[1]) or abs(df_dt[0]) == INF or abs(df_dt[1]) == INF
        if bad_dt or time_err >= f32(delta) or not children:
            time_err, enq = f32(0), True
    else:
        f = f32(-1) if F[1] <= 0 else f32(1)
    return time_err, fast, f, enq


def _by_key(cells):
    return {(int(c["level"]), int(c["ix"]), int(c["iy"]), int(c["iz"])): c for c in cells}


@pytest.mark.parametrize("lipschitz", [1, 0])
@pytest.mark.parametrize("text", [scenes.spheres16(0), scenes.csg(24, 3, 0.9)], ids=["spheres16", "csg24"])
def test_cells_match_restatement(text, lipschitz):
    """Every cell of levels 3 and 4 that a frame evaluates, frames at t = 0,
    1/60 and 2/60 of a localsubdiv-6 octree (time_err accumulating over
    frames, cells reused or re-enqueued, parents turning fast)."""
    oracle.build()
    tape = api.IR.new(text).gpu_instructions
    delta = 0.01
    p = api.default_params(localsubdiv=6, pointsample=0, lipschitz_corrected=lipschitz, delta=delta)
    S = oracle.Scene(tape, p)
    times = [f32(0.0), f32(1.0 / 60.0), f32(2.0 / 60.0)]
    S.invert(float(times[0]))
    prev = _by_key(S.cells())
    checked = accumulated = 0
    for t1 in times[1:]:
        S.invert(float(t1))
        now = _by_key(S.cells())
        todo = [k for k, c in now.items() if k[0] in (3, 4) and c["t"] == t1]
        boxes = np.zeros((len(todo), 8), f32)
        meta = []
        for n, k in enumerate(todo):
            c = now[k]
            parent = now[(k[0] - 1, k[1] // 2, k[2] // 2, k[3] // 2)]
            old = prev.get(k)
            new = old is None
            point = new or parent["fast"] == 1.0  # width > epsilon at these levels
            t0 = t1 if point else f32(old["t"])
            boxes[n, 0:2], boxes[n, 2:4], boxes[n, 4:6] = c["x"], c["y"], c["z"]
            boxes[n, 6:8] = (min(t0, t1), max(t0, t1))
            meta.append((k, point, new, old))
        out = oracle.eval_boxes(tape, boxes, reverse=True)
        for n, (k, point, new, old) in enumerate(meta):
            c = now[k]
            F = (f32(out[n, 0]), f32(out[n, 1]))
            if point:  # no reverse pass: df stays 0, the cell's fast flag is cleared
                te = f32(0) if new else f32(old["time_err"])
                fast = f32(0)
                if F[0] <= 0 <= F[1]:
                    f = f32(0)
                    te = f32(0)  # a point time range always re-enqueues (4018)
                else:
                    f = f32(-1) if F[1] <= 0 else f32(1)
            else:
                sens = [(f32(out[n, 2 + 2 * q]), f32(out[n, 3 + 2 * q])) for q in range(4)]
                te, fast, f, _ = cell_update(F, sens, old["t"], t1, delta, f32(old["time_err"]),
                                             bool(old["has_children"]), lipschitz)
                accumulated += int(te != 0)
            assert (c["f"], c["time_err"], c["fast"]) == (f, te, fast), (t1, k, point, (c["f"], c["time_err"],
                                                                                     c["fast"]), (f, te, fast))
            checked += 1
        prev = now
    assert checked > 100 and accumulated > 10, (checked, accumulated)


@pytest.mark.parametrize("text", [scenes.spheres16(0), scenes.csg(24, 3, 0.9)], ids=["spheres16", "csg24"])
def test_point_sampled_leaves_match_restatement(text):
    """Leaves (width <= epsilon) with point sampling (compute.wgsl:3603-3621,
    4011-4045): evaluated at the current time at the midpoint (lo + hi) / 2
    of their box, f from the sign of that value (0 only where it is 0), never
    re-enqueued, fast cleared, time_err and the normal kept from the cell's
    previous life (0 for a new cell: no derivative is taken at a point
    time).  Every leaf of two frames of a localsubdiv-6 octree."""
    oracle.build()
    tape = api.IR.new(text).gpu_instructions
    L = 6
    p = api.default_params(localsubdiv=L, pointsample=1, lipschitz_corrected=1, delta=0.01)
    S = oracle.Scene(tape, p)
    prev = {}
    checked = 0
    for t in (f32(0.0), f32(1.0 / 60.0)):
        S.invert(float(t))
        now = _by_key(S.cells())
        leaves = [k for k, c in now.items() if k[0] == L and c["t"] == t]
        boxes = np.zeros((len(leaves), 8), f32)
        for n, k in enumerate(leaves):
            c = now[k]
            for a, ax in enumerate("xyz"):
                boxes[n, 2 * a: 2 * a + 2] = f32(f32(c[ax][0] + c[ax][1]) / f32(2))  # MID, 2510-2512
            boxes[n, 6:8] = t
        out = oracle.eval_boxes(tape, boxes, reverse=False)
        for n, k in enumerate(leaves):
            c, old = now[k], prev.get(k)
            F = (f32(out[n, 0]), f32(out[n, 1]))
            f = f32(0) if F[0] <= 0 <= F[1] else (f32(-1) if F[1] <= 0 else f32(1))
            te = f32(0) if old is None else f32(old["time_err"])
            nrm = (f32(0), f32(0), f32(0)) if old is None else (old["dx"], old["dy"], old["dz"])
            assert (c["f"], c["fast"], c["time_err"], c["has_children"]) == (f, f32(0), te, 0), (t, k)
            assert (c["dx"], c["dy"], c["dz"]) == nrm, (t, k)
            checked += 1
        prev = now
    assert checked > 200, checked


def _temporal_bound(F, sens, t0, t1, delta, lipschitz):
    """|df| clamped to [0, delta] as time_err's increment (3971-3996) and df_dt."""
    df_dt = sens[3]
    dt = f32(f32(t1) - f32(t0))
    df = mul_if(df_dt[0], df_dt[1], dt)
    W = mul_if(f32(-1), f32(1), f32(F[1] - F[0]))
    df = (INF, -INF) if (df[1] < W[0] or W[1] < df[0]) else (max(df[0], W[0]), min(df[1], W[1]))
    if lipschitz and abs_i(*df)[1] != 0:
        s = [sqr_i(*sens[q]) for q in range(3)]
        acc = (f32(s[1][0] + s[2][0]), f32(s[1][1] + s[2][1]))
        acc = (f32(s[0][0] + acc[0]), f32(s[0][1] + acc[1]))
        lb = abs_i(np.sqrt(max(acc[0], f32(0))), np.sqrt(max(acc[1], f32(0))))[0]
        if not np.isnan(lb):
            q = [f32(df[0] / lb), f32(df[1] / lb)]
            df = (min(q), max(q))
    if df[0] == -INF or df[1] == INF or np.isnan(df[0]) or np.isnan(df[1]):
        df = (f32(delta), f32(delta))
    return np.clip(abs_i(*df)[1], f32(0), f32(delta)), df_dt


@pytest.mark.parametrize("lipschitz", [0, 1])
def test_swept_volume_cells_match_restatement(lipschitz):
    """Swept volume (compute.wgsl:3603-3605, 3629, 4028-4044): a cell's time
    range is [t0, t] when new or at most epsilon wide, else [its last time,
    t]; interior cells with children are skipped; an empty cell keeps its f
    (1 when new, mallocV 3444), full cells turn -1, ambiguous 0 with the
    re-enqueue rule; no fast flag; nothing is ever deallocated.  Every cell
    of four frames [k/16, (k+1)/16] of a localsubdiv-5 octree of rotating
    primitives."""
    with np.errstate(all="ignore"):
        oracle.build()
        tape = api.IR.new(scenes.swept(8, 4)).gpu_instructions
        delta, L = 0.01, 5
        p = api.default_params(localsubdiv=L, pointsample=0, swept_volume=1, lipschitz_corrected=lipschitz,
                               delta=delta)
        eps = f32(10.0 * 2.0 ** -L)
        S = oracle.Scene(tape, p)
        prev = {}
        checked = skipped = 0
        for k in range(4):
            t0, t1 = f32(k / 16.0), f32((k + 1) / 16.0)
            S.invert(float(t1), float(t0))
            now = _by_key(S.cells())
            assert set(prev) <= set(now), "a swept-volume cell was deallocated"
            todo = [key for key, c in now.items() if key[0] >= 1 and c["t"] == t1]
            boxes = np.zeros((len(todo), 8), f32)
            meta = []
            for n, key in enumerate(todo):
                c, old = now[key], prev.get(key)
                width = f32(c["x"][1] - c["x"][0])
                lo = t0 if (old is None or width <= eps) else f32(old["t"])
                boxes[n, 0:2], boxes[n, 2:4], boxes[n, 4:6] = c["x"], c["y"], c["z"]
                boxes[n, 6:8] = (min(lo, t1), max(lo, t1))
                meta.append((key, old, width, lo))
            out = oracle.eval_boxes(tape, boxes, reverse=True)
            for n, (key, old, width, lo) in enumerate(meta):
                c = now[key]
                if old is not None and old["f"] < 0 and old["has_children"]:  # interior: skipped (3629)
                    assert (c["f"], c["time_err"]) == (old["f"], old["time_err"]), key
                    skipped += 1
                    continue
                F = (f32(out[n, 0]), f32(out[n, 1]))
                sens = [(f32(out[n, 2 + 2 * q]), f32(out[n, 3 + 2 * q])) for q in range(4)]
                inc, df_dt = _temporal_bound(F, sens, lo, t1, delta, lipschitz)
                te = f32((f32(0) if old is None else f32(old["time_err"])) + inc)
                f_old = f32(1) if old is None else f32(old["f"])
                if F[0] <= 0 <= F[1]:
                    f = f32(0)
                    bad = any(np.isnan(v) or abs(v) == INF for v in df_dt)
                    if width > eps and (old is None or bad or lo == t1 or te >= f32(delta)
                                        or not old["has_children"]):
                        te = f32(0)
                else:
                    f = f32(-1) if F[1] <= 0 else f_old
                mids = tuple(f32(f32(sens[q][0] + sens[q][1]) / f32(2)) for q in range(3))
                assert (c["f"], c["time_err"], c["fast"]) == (f, te, f32(0)), (k, key, (c["f"], c["time_err"]),
                                                                                (f, te))
                assert (c["dx"], c["dy"], c["dz"]) == mids, key
                checked += 1
            prev = now
        assert checked > 500, (checked, skipped)
