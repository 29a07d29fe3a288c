"""The float64 point evaluator used by the rigour tests agrees with the
oracle's round-to-nearest interval evaluation on degenerate (point) boxes,
to float32 accuracy.  No device needed."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from point_eval import evaluate
from temporalsetinversion_b200 import api, scenes


@pytest.mark.parametrize("text", [scenes.spheres16(0), scenes.csg(24, 3, 0.9), scenes.swept(8, 4)],
                         ids=["spheres16", "csg24", "swept8"])
def test_point_eval_matches_oracle(text):
    oracle.build()
    tape = api.IR.new(text).gpu_instructions
    rng = np.random.default_rng(5)
    pts = rng.uniform(-1.2, 1.2, (256, 4)).astype(np.float32)
    pts[:, 3] = rng.uniform(0, 1, 256).astype(np.float32)
    boxes = np.repeat(pts, 2, axis=1)  # [x, x, y, y, z, z, t, t]
    got = oracle.eval_boxes(tape, boxes, reverse=False)[:, 0]
    want = evaluate(tape, pts[:, 0], pts[:, 1], pts[:, 2], pts[:, 3])
    assert np.allclose(got, want, rtol=1e-4, atol=1e-5)
