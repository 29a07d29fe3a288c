"""Regenerate the golden fixtures under tests/golden/.

  tapes/<scene>.json  — the reference's four scene files (scenes/*.ll of the
                        reference checkout) lowered by oracle/ir_ref.py, the
                        pure-Python restatement of src/ir.rs, in the 32-byte
                        GPUInstruction layout (literals as f32 bit patterns).
  oracle_cases.json   — summaries (counters and a SHA-256 of the sorted cell
                        records) of CPU-oracle runs on small cases, and
                        SHA-256s of a 64x36 trace of each final octree
                        (depth, normal, rgba), so that a change to the
                        oracle is caught and the device path can be checked
                        against them without running the oracle.

Run from the repository root with the reference checkout available:
    python tests/golden/make_golden.py [/path/to/reference]
The GPU tests read only the committed JSON, never the reference checkout.
"""
from __future__ import annotations

import hashlib
import json
import os
import math
import struct
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import ir_ref  # noqa: E402

HERE = Path(__file__).resolve().parent
SCENES = ["cables", "cradle", "piano", "sponza"]


def f32_bits(x: float) -> str:
    return "%08x" % struct.unpack("<I", struct.pack("<f", x))[0]


def write_tapes(ref_root: Path) -> None:
    for name in SCENES:
        text = (ref_root / "scenes" / (name + ".ll")).read_text()
        rows = ir_ref.lower(text, 0.0)
        out = {
            "source": "scenes/%s.ll lowered by ir.rs:190-366 (restated in oracle/ir_ref.py)" % name,
            "instruction_count": len(rows),
            "instructions": [[r[0], r[1], r[2], f32_bits(r[3]), f32_bits(r[4]), f32_bits(r[5])] for r in rows],
        }
        (HERE / "tapes" / (name + ".json")).write_text(json.dumps(out, separators=(",", ":")) + "\n")


def load_tape(name: str) -> np.ndarray:
    from temporalsetinversion_b200.api import GPU_INSTR_DTYPE
    d = json.loads((HERE / "tapes" / (name + ".json")).read_text())
    arr = np.zeros(len(d["instructions"]), dtype=GPU_INSTR_DTYPE)
    for i, r in enumerate(d["instructions"]):
        arr[i]["index_"], arr[i]["opcode_uses"], arr[i]["larg_rarg"] = r[0], r[1], r[2]
        arr[i]["literal"] = struct.unpack("<f", bytes.fromhex(r[3])[::-1])[0]
        arr[i]["val"][0] = struct.unpack("<f", bytes.fromhex(r[4])[::-1])[0]
        arr[i]["val"][1] = struct.unpack("<f", bytes.fromhex(r[5])[::-1])[0]
    return arr


def cells_digest(cells: np.ndarray) -> str:
    order = np.lexsort((cells["iz"], cells["iy"], cells["ix"], cells["level"]))
    return hashlib.sha256(cells[order].tobytes()).hexdigest()


def oracle_cases():
    """(case name, tape source, params, frame times)"""
    from temporalsetinversion_b200 import scenes
    cases = [
        ("spheres16_L6", ("gen", scenes.spheres16(0)), dict(localsubdiv=6, pointsample=0), [0.0, 1 / 60, 2 / 60]),
        ("csg24_L6_lip", ("gen", scenes.csg(24, 3)), dict(localsubdiv=6, lipschitz_corrected=1, pointsample=1),
         [0.0, 0.05, 0.1, 0.15]),
        ("swept8_L5", ("gen", scenes.swept(8, 4)), dict(localsubdiv=5, swept_volume=1), [0.25, 0.5, 0.75]),
        # cinematic path tracing (two bounces, shadow rays, sky) with tape normals
        ("spheres16_L6_cinematic", ("gen", scenes.spheres16(0)),
         dict(localsubdiv=6, pointsample=0, cinematic=1, fast_normals=1, samples=2, see_background=1), [0.0, 1 / 60]),
    ]
    for name in SCENES:
        cases.append(("%s_L5" % name, ("tape", name), dict(localsubdiv=5), [0.0, 1 / 60]))
    return cases


IMAGE_EYE = (0.3, 0.6, 2.5)
IMAGE_RES = (64, 36)


def image_digests(img: dict) -> dict:
    out = {k: hashlib.sha256(np.ascontiguousarray(img[k], dtype=np.float32).tobytes()).hexdigest()
           for k in ("depth", "normal", "rgba")}
    out["hits"] = int((img["depth"] >= 0).sum())
    return out


def case_tape(case):
    from temporalsetinversion_b200 import api
    _, (kind, src), _, _ = case
    return api.IR.new(src).gpu_instructions if kind == "gen" else load_tape(src)


def image_uniforms(case):
    from temporalsetinversion_b200 import api, scenes
    return api.make_uniforms(scenes.camera_look_at(IMAGE_EYE), IMAGE_RES, case[3][-1])


def run_case(case):
    import oracle
    from temporalsetinversion_b200 import api
    name, _, params, times = case
    tape = case_tape(case)
    p = api.default_params(**params)
    S = oracle.Scene(tape, p)
    frames = [S.invert(t) for t in times]
    cells = S.cells()
    return {"frames": frames, "cells": int(len(cells)), "digest": cells_digest(cells),
            "image": image_digests(S.trace(image_uniforms(case)))}


def main() -> None:
    # the reference checkout: the first argument, else TSI_REFERENCE_DIR, else
    # a `reference` folder beside this repository
    default = os.environ.get("TSI_REFERENCE_DIR", str(ROOT.parent / "reference"))
    ref = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(default)
    if (ref / "scenes").exists():
        write_tapes(ref)
    results = {case[0]: run_case(case) for case in oracle_cases()}
    (HERE / "oracle_cases.json").write_text(json.dumps(results, indent=1, sort_keys=True) + "\n")
    print("wrote", len(results), "oracle cases")


if __name__ == "__main__":
    main()
