"""The oracle against its committed fixtures (tests/golden/oracle_cases.json,
made by tests/golden/make_golden.py): frame counters, the SHA-256 of the
sorted cell records and of a 64x36 trace (depth, normal, rgba) for each
small case, the four reference scene tapes among them.  A change to the
oracle's arithmetic shows up here before it can move the device parity
tests' reference."""
from __future__ import annotations

import json
from pathlib import Path

import pytest

import oracle
from golden.make_golden import oracle_cases, run_case

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "oracle_cases.json").read_text())
CASES = {c[0]: c for c in oracle_cases()}


def test_every_case_has_a_fixture():
    assert sorted(CASES) == sorted(GOLDEN)


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_fixture(name):
    oracle.build()
    got = run_case(CASES[name])
    want = GOLDEN[name]
    assert got["frames"] == want["frames"]
    assert (got["cells"], got["digest"]) == (want["cells"], want["digest"])
    assert got["image"] == want["image"]
    assert want["image"]["hits"] > 50
