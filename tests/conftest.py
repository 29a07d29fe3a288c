"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 (B200) device")


@pytest.fixture(scope="session")
def device():
    """One tsi_ctx for the session.  A GPU test without a device fails (the
    library has no CPU fallback to hide behind)."""
    from temporalsetinversion_b200 import Device
    dev = Device()
    yield dev
    dev.close()


def sorted_cells(c: np.ndarray) -> np.ndarray:
    return c[np.lexsort((c["iz"], c["iy"], c["ix"], c["level"]))]


def same_values(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Elementwise float equality where NaN == NaN and -0 == +0."""
    return (a == b) | (np.isnan(a) & np.isnan(b))


CELL_FIELDS = ["f", "t", "time_err", "fast", "has_children", "x", "y", "z", "dx", "dy", "dz"]


def assert_cells_equal(got: np.ndarray, ref: np.ndarray, fields=CELL_FIELDS) -> None:
    g, r = sorted_cells(got), sorted_cells(ref)
    assert len(g) == len(r), "cell count differs: gpu %d oracle %d" % (len(g), len(r))
    for k in ("level", "ix", "iy", "iz"):
        assert np.array_equal(g[k], r[k]), "cell keys differ"
    for k in fields:
        ok = same_values(g[k], r[k]) if g[k].dtype.kind == "f" else (g[k] == r[k])
        if not np.all(ok):
            bad = np.nonzero(~ok.reshape(len(g), -1).all(axis=1))[0]
            i = int(bad[0])
            raise AssertionError("field %s differs in %d cells; first at key %s: gpu %r oracle %r" % (
                k, len(bad), tuple(int(g[q][i]) for q in ("level", "ix", "iy", "iz")), g[k][i], r[k][i]))
