"""The device path against the committed oracle fixtures
(tests/golden/oracle_cases.json) without running the oracle: per small case
(generated scenes and the reference's four scene tapes) the frame counters,
the SHA-256 of the sorted cell records and of a 64x36 trace's depth, normal
and rgba images."""
from __future__ import annotations

import json
from pathlib import Path

import pytest

from golden.make_golden import case_tape, cells_digest, image_digests, image_uniforms, oracle_cases
from temporalsetinversion_b200 import Scene, Tape, api

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "oracle_cases.json").read_text())
CASES = {c[0]: c for c in oracle_cases()}
COUNTERS = ["parents_expanded", "cells_evaluated", "cells_reverse", "cells_ambiguous", "cells_empty", "cells_full",
            "cells_enqueued", "cells_reused"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_device_matches_fixture(device, name):
    case = CASES[name]
    want = GOLDEN[name]
    s = Scene(device, Tape.upload(device, case_tape(case)), api.default_params(**case[2]), voxel_capacity=1 << 20)
    for t, wf in zip(case[3], want["frames"]):
        st = s.invert(t).as_dict()
        assert {k: st[k] for k in COUNTERS} == {k: wf[k] for k in COUNTERS}, t
    cells = s.cells()
    assert (len(cells), cells_digest(cells)) == (want["cells"], want["digest"])
    assert image_digests(s.trace(image_uniforms(case))) == want["image"]
    s.close()
