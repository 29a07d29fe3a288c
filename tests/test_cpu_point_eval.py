"""The float64 point evaluator used by the rigour tests agrees with the
oracle's round-to-nearest interval evaluation on degenerate (point) boxes,
to float32 accuracy.  No device needed."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from point_eval import evaluate
from golden.make_golden import load_tape
from temporalsetinversion_b200 import api, scenes


@pytest.mark.parametrize("src", ["spheres16", "csg24", "swept8", "cables", "cradle", "piano", "sponza"])
def test_point_eval_matches_oracle(src):
    """Generated scenes and the reference's four scene tapes (cables has sin,
    cos, exp and the operand-swapped atan2)."""
    oracle.build()
    gen = {"spheres16": lambda: scenes.spheres16(0), "csg24": lambda: scenes.csg(24, 3, 0.9),
           "swept8": lambda: scenes.swept(8, 4)}
    tape = api.IR.new(gen[src]()).gpu_instructions if src in gen else load_tape(src)
    rng = np.random.default_rng(5)
    pts = rng.uniform(-1.2, 1.2, (256, 4)).astype(np.float32)
    pts[:, 3] = rng.uniform(0, 1, 256).astype(np.float32)
    boxes = np.repeat(pts, 2, axis=1)  # [x, x, y, y, z, z, t, t]
    got = oracle.eval_boxes(tape, boxes, reverse=False)[:, 0]
    want = evaluate(tape, pts[:, 0], pts[:, 1], pts[:, 2], pts[:, 3])
    assert np.allclose(got, want, rtol=1e-4, atol=1e-5)
