"""Test helper: the temporal guarantee of cells carried over between frames.

A cell classified empty (f = +1) or full (f = -1) at time t_e and not
re-evaluated since keeps its sign up to the field change since t_e.  That
change is covered by the time_err of its ancestors: the parent was
re-enqueued at t_e (time_err reset, compute.wgsl:4016-4025) and every later
evaluation of an ancestor adds a bound of the change over [its last
evaluation, now] on its whole box (3971-3996), until it is re-enqueued,
which re-evaluates its children.  So at every point p of the cell and time
t, sign * f(p, t) >= -G * (sum of the ancestors' time_err), with G = 1 in
field units (lipschitz_corrected off) or, with the correction (time_err in
distance units), G a bound of |grad f| over the cell: 1 for the signed
distance scenes used here."""
from __future__ import annotations

import numpy as np

from point_eval import evaluate


def ancestors_time_err(cells: np.ndarray, sel: np.ndarray) -> np.ndarray:
    """Per cell of `sel`, the sum of time_err over its ancestors below the root."""
    te = {(int(c["level"]), int(c["ix"]), int(c["iy"]), int(c["iz"])): float(c["time_err"]) for c in cells}
    out = np.zeros(len(sel))
    for i, c in enumerate(sel):
        l, x, y, z = int(c["level"]), int(c["ix"]), int(c["iy"]), int(c["iz"])
        s = 0.0
        while l > 1:
            l, x, y, z = l - 1, x // 2, y // 2, z // 2
            s += te[(l, x, y, z)]
        out[i] = s
    return out


def samples(cells: np.ndarray, rng, n_random: int = 8) -> np.ndarray:
    """Corners, centre and random interior points of every cell box."""
    lo = np.stack([cells["x"][:, 0], cells["y"][:, 0], cells["z"][:, 0]], axis=1).astype(np.float64)
    hi = np.stack([cells["x"][:, 1], cells["y"][:, 1], cells["z"][:, 1]], axis=1).astype(np.float64)
    corners = np.array([[(k >> 0) & 1, (k >> 1) & 1, (k >> 2) & 1] for k in range(8)], np.float64)
    u = np.concatenate([corners, [[0.5, 0.5, 0.5]], rng.uniform(size=(n_random, 3))], axis=0)
    return lo[:, None, :] + u[None, :, :] * (hi - lo)[:, None, :]


def carried_excursions(tape, cells: np.ndarray, t: float, rng) -> tuple:
    """For the carried-over empty/full cells of `cells` at time t: how far f
    reaches into the other sign at float64 samples, and the ancestors' bound."""
    car = cells[(cells["t"] < np.float32(t)) & (cells["f"] != 0)]
    if len(car) == 0:
        return np.zeros(0), np.zeros(0)
    pts = samples(car, rng)
    f = evaluate(tape, pts[..., 0], pts[..., 1], pts[..., 2], np.float64(np.float32(t)))
    return -(car["f"][:, None].astype(np.float64) * f).min(axis=1), ancestors_time_err(cells, car)
