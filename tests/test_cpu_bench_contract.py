"""bench.py's reference arm on the CPU: one JSON line with the keys of the
benchmark contract (the device arm prints the same keys plus its roofline,
clocks and launch count, on a GPU)."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["n_gpus"] == 1 and line["value"] > 0
    assert line["unit"] == "frames/s" and line["higher_is_better"] is True
    assert line["config"]["workload"] == "csg256_L10_1080p_120f"
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["cores"] >= 1 and cb["kind"] == "port" and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_runs_without_the_product_library():
    """The reference arm lowers its tape with the oracle's ir.rs restatement
    and builds its parameters itself: libtsi.so is never loaded."""
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3'];"
            "runpy.run_path('bench.py', run_name='__main__');"
            "maps = open('/proc/self/maps').read();"
            "print('LIBTSI_LOADED' if 'libtsi.so' in maps else 'LIBTSI_ABSENT')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    assert "LIBTSI_ABSENT" in r.stdout and "LIBTSI_LOADED" not in r.stdout


def test_reference_params_equal_library_defaults():
    sys.path.insert(0, str(ROOT))
    import bench
    from temporalsetinversion_b200 import api
    a, b = bench.reference_params(localsubdiv=10, delta=0.01), api.default_params(localsubdiv=10, delta=0.01)
    assert bytes(a) == bytes(b)
