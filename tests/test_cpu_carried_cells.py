"""The temporal guarantee of carried-over cells, on the oracle (round to
nearest, the reference's semantics): every empty or full cell not
re-evaluated this frame keeps its sign up to its ancestors' accumulated
time_err (tests/carried_ref.py), at float64 samples over 40 frames.

With lipschitz_corrected on, the reference's time_err is df / lb, lb the
lower end of |sqrt(sum sens^2)| over the cell (compute.wgsl:3980-3992).
Its MIN/MAX reverse rule gives (1, 1) for overlapping operands
(2885-2903), so both branches' gradients add up and lb can exceed the
true |grad f| (1 for a signed distance): the corrected time_err then
undercounts the field change and a carried cell can cross by more than its
ancestors' time_err.  The second test records one such case.  The device's
directed-rounding mode takes the hull [0, 1] instead and keeps the bound
(tests/test_gpu_rigour.py)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from carried_ref import carried_excursions
from temporalsetinversion_b200 import api, scenes

CASES = {
    "spheres16_d0.03": (lambda: scenes.spheres16(0), 0.03),
    "csg24_d0.01": (lambda: scenes.csg(24, 3, 0.9), 0.01),
    "csg64_d0.03": (lambda: scenes.csg(64, 5, 0.85), 0.03),
}


def _run(text, delta, lipschitz, frames=40):
    oracle.build()
    tape = api.IR.new(text).gpu_instructions
    p = api.default_params(localsubdiv=6, pointsample=0, lipschitz_corrected=lipschitz, delta=delta)
    S = oracle.Scene(tape, p)
    rng = np.random.default_rng(1)
    exc, bound = [], []
    for k in range(frames):
        t = k / 60.0
        S.invert(t)
        e, b = carried_excursions(tape, S.cells(), t, rng)
        exc.append(e)
        bound.append(b)
    return np.concatenate(exc), np.concatenate(bound)


@pytest.mark.parametrize("case", sorted(CASES))
def test_carried_cells_stay_within_ancestors_time_err(case):
    make, delta = CASES[case]
    exc, bound = _run(make(), delta, 0)
    assert len(exc) > 50, len(exc)
    over = exc > bound + 1e-6
    assert not over.any(), "%d carried cells cross by more than their ancestors' time_err, e.g. %g > %g" % (
        over.sum(), exc[over][0], bound[over][0])
    if case.startswith("csg"):  # the surface did move into carried cells
        assert (exc > 0).any()


def test_lipschitz_time_err_undercounts_with_the_reference_min_max_rule():
    exc, bound = _run(scenes.csg(64, 5, 0.85), 0.03, 1)
    over = exc > bound + 1e-6
    assert over.any()
    assert np.max(exc[over] / bound[over]) < 2.0  # about 1.3 here
