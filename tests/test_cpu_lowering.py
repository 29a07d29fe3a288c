"""Tape lowering (src/ir.rs:140-366) in the C ABI library against the
pure-Python restatement in oracle/ir_ref.py and the golden tapes of the
reference's four scene files.  No device needed."""
from __future__ import annotations

import ctypes as C
import os
import re
import struct
from pathlib import Path

import numpy as np
import pytest

import ir_ref  # noqa: F401  (oracle/ on sys.path below)
from golden.make_golden import load_tape
from temporalsetinversion_b200 import _native as N, api, scenes

ROOT = Path(__file__).resolve().parents[1]
# the reference checkout: TSI_REFERENCE_DIR, else a `reference` folder beside
# this repository; the tests that read its scene files skip without it
REF = Path(os.environ.get("TSI_REFERENCE_DIR", str(ROOT.parent / "reference")))
FIXTURE_COUNTS = {"cables": 297, "cradle": 329, "piano": 325, "sponza": 307}


def lower(text: str, time: float = 0.0) -> np.ndarray:
    return api.IR.new(text, time).gpu_instructions


def as_tuples(arr):
    return [(int(r["index_"]), int(r["opcode_uses"]), int(r["larg_rarg"]),
             struct.pack("<f", r["literal"]), float(r["val"][0]), float(r["val"][1])) for r in arr]


def ref_tuples(rows):
    return [(r[0], r[1], r[2], struct.pack("<f", r[3]), r[4], r[5]) for r in rows]


def test_library_loads_and_exports_every_header_symbol():
    lib = N.load()
    header = (ROOT / "include" / "tsi.h").read_text()
    names = re.findall(r"TSI_API\s+[^;(]*?\b(tsi_\w+)\s*\(", header)
    assert len(names) == len(set(names)) and len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
        assert name in N.SIGNATURES, "binding missing for %s" % name
    assert lib.tsi_version() == 1


def test_rust_binding_declares_the_public_header():
    """rust/tsi-sys declares every entry point above the header's
    diagnostics block, and nothing the header lacks."""
    header = (ROOT / "include" / "tsi.h").read_text()
    public = header.split("---------------- diagnostics")[0]
    names = set(re.findall(r"TSI_API\s+[^;(]*?\b(tsi_\w+)\s*\(", public))
    rust = (ROOT / "rust" / "tsi-sys" / "src" / "lib.rs").read_text()
    declared = set(re.findall(r"pub fn (tsi_\w+)\s*\(", rust))
    all_names = set(re.findall(r"TSI_API\s+[^;(]*?\b(tsi_\w+)\s*\(", header))
    assert names - declared == set()
    assert declared - all_names == set()


@pytest.mark.parametrize("scene", sorted(FIXTURE_COUNTS))
def test_golden_tapes(scene):
    tape = load_tape(scene)
    assert len(tape) == FIXTURE_COUNTS[scene]
    # four ARG slots with the root box (ir.rs:335-348), RET last
    for i in range(4):
        assert (tape[i]["opcode_uses"] >> 16) & 0x3FFF == 1 + i
        assert (tape[i]["opcode_uses"] >> 30) == 3
    assert list(tape[0]["val"]) == [-5.0, 5.0]
    assert (tape[-1]["opcode_uses"] >> 16) & 0x3FFF == 28


@pytest.mark.skipif(not (REF / "scenes").exists(), reason="reference checkout not mounted")
@pytest.mark.parametrize("scene", sorted(FIXTURE_COUNTS))
def test_cpp_lowering_matches_restatement_on_reference_scenes(scene):
    text = (REF / "scenes" / (scene + ".ll")).read_text()
    got = as_tuples(lower(text))
    assert got == ref_tuples(ir_ref.lower(text))
    assert got == as_tuples(load_tape(scene))


@pytest.mark.parametrize("gen", ["spheres16", "csg256", "swept64", "csg8"])
def test_cpp_lowering_matches_restatement_on_generated(gen):
    text = {"spheres16": scenes.spheres16(0), "csg256": scenes.csg(256, 1), "swept64": scenes.swept(64, 2),
            "csg8": scenes.csg(8, 5)}[gen]
    assert as_tuples(lower(text, 0.25)) == ref_tuples(ir_ref.lower(text, 0.25))


HDR = "define dso_local float @_Z1fffff(float %0, float %1, float %2, float %3) local_unnamed_addr #5 {\n"


def test_encoding_details():
    text = HDR + "\n".join([
        "  %5 = fmul float %0, %0",                      # SQR rewrite, one use of x
        "  %6 = fsub float 0x3FF8000000000000, %5",      # literal left: op_top 2
        "  %7 = fadd float %6, 2.500000e-01",            # literal right: op_top 1
        "  %8 = tail call float @llvm.maxnum.f32(float %7, float %1) #10",  # op_top 0
        "  %9 = fneg float %8",
        "  ret float %9",
    ]) + "\n}\n"
    g = lower(text)
    op = lambda i: (g[i]["opcode_uses"] >> 16) & 0x3FFF
    top = lambda i: g[i]["opcode_uses"] >> 30
    uses = lambda i: g[i]["opcode_uses"] & 0xFFFF
    assert len(g) == 10
    assert op(4) == 11 and top(4) == 1 and g[4]["larg_rarg"] == 0 << 16  # SQR of x
    assert uses(0) == 1 and uses(1) == 1 and uses(2) == 0 and uses(3) == 0
    assert op(5) == 6 and top(5) == 2 and g[5]["larg_rarg"] == 4 and g[5]["literal"] == 1.5
    assert op(6) == 5 and top(6) == 1 and g[6]["larg_rarg"] == (5 << 16) and g[6]["literal"] == 0.25
    assert op(7) == 18 and top(7) == 0 and g[7]["larg_rarg"] == ((6 << 16) | 1)
    assert op(8) == 16 and top(8) == 1
    assert op(9) == 28 and uses(9) == 1  # dummy use of the last instruction (ir.rs:355)
    assert [int(g[i]["index_"]) for i in range(10)] == list(range(10))


@pytest.mark.parametrize("bad", [
    "no function here",
    HDR + "  %5 = fcmp olt float %0, %1\n  ret float %5\n}\n",
    HDR + "  %5 = fadd float %0, %9\n  ret float %5\n}\n",           # forward reference
    HDR + "  %5 = tail call float @tanf(float %0) #10\n  ret float %5\n}\n",
    HDR + "\n  ret float %0\n}\n",                                     # empty line
    HDR + "  %5 = tail call float @llvm.minnum.f32(float 1.0, float %0) #10\n  ret float %5\n}\n",
])
def test_parse_errors_where_ir_rs_panics(bad):
    lib = N.load()
    raw = bad.encode()
    n = C.c_uint32(0)
    assert lib.tsi_ir_lower(raw, len(raw), 0.0, None, 0, C.byref(n)) == 2
    with pytest.raises(ValueError):
        ir_ref.lower(bad)


def _simulate_registers(text):
    """Replays the register allocation: every operand read must find the SSA
    value it names in its register (no clobbering)."""
    lib = N.load()
    raw = text.encode()
    info = N.TapeInfo()
    n = len(api.IR.new(text).gpu_instructions)
    slot_reg = (C.c_uint32 * n)()
    assert lib.tsi_ir_tape_info(raw, len(raw), C.byref(info), slot_reg, n) == 0
    g = api.IR.new(text).gpu_instructions
    holder = {}
    for j in range(4):
        holder[slot_reg[j]] = j
    for j in range(4, n):
        top = g[j]["opcode_uses"] >> 30
        l, r = g[j]["larg_rarg"] >> 16, g[j]["larg_rarg"] & 0xFFFF
        reads = ([l] if top in (0, 1) else []) + ([r] if top in (0, 2) else [])
        for s in reads:
            assert holder.get(slot_reg[s]) == s, "slot %d reads slot %d from a clobbered register" % (j, s)
        holder[slot_reg[j]] = j
    assert slot_reg[n - 1] == info.reserved
    return info


@pytest.mark.parametrize("gen", ["spheres16", "csg256", "swept64"])
def test_register_allocation_never_clobbers(gen):
    text = {"spheres16": scenes.spheres16(0), "csg256": scenes.csg(256, 1), "swept64": scenes.swept(64, 2)}[gen]
    info = _simulate_registers(text)
    assert info.registers <= 32


@pytest.mark.skipif(not (REF / "scenes").exists(), reason="reference checkout not mounted")
@pytest.mark.parametrize("scene", sorted(FIXTURE_COUNTS))
def test_register_allocation_reference_scenes(scene):
    _simulate_registers((REF / "scenes" / (scene + ".ll")).read_text())


def test_packed_handlers_and_flags():
    lib = N.load()
    text = HDR + "\n".join([
        "  %5 = fadd float 0x3FF8000000000000, %0",   # ADD with a literal left: unsupported -> BAD_FI
        "  %6 = tail call float @fmodf(float %5, float %1) #10",  # MOD_II
        "  %7 = tail call float @atan2f(float %6, float 2.000000e+00) #10",  # ATAN2_IF
        "  ret float %7",
    ]) + "\n}\n"
    g = api.IR.new(text).gpu_instructions
    words = (C.c_uint32 * 16)()
    info = N.TapeInfo()
    assert lib.tsi_compile_gpu_instructions(g.ctypes.data_as(C.POINTER(N.GPUInstruction)), len(g), words, 16,
                                            C.byref(info)) == 0
    h = [words[2 * i] & 63 for i in range(4)]
    assert h == [33, 9, 20, 1]  # H_BAD_FI, H_MOD_II, H_ATAN2_IF, H_COPY
    assert (words[0] >> 6) & 1 == 1  # x used once
    assert struct.unpack("<f", struct.pack("<I", words[5]))[0] == 2.0


def test_frame_dump_png(tmp_path):
    """rt_main's f32 frame as the reference's 8-bit PNG dump (main.rs:692-715):
    clamp to [0, 1], scale by 255, round; the file decodes back to it."""
    import zlib

    rgba = np.array([[[0.0, 1.0, 0.5, 2.0], [-1.0, np.nan, 0.25, 1.0 / 510.0]]], np.float32)
    px = api.rgba8(rgba)
    assert px.tolist() == [[[0, 255, 128, 255], [0, 0, 64, 1]]]
    path = tmp_path / "frame.png"
    api.save_png(path, rgba)
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    i = data.index(b"IDAT")
    n = struct.unpack(">I", data[i - 4:i])[0]
    raw = zlib.decompress(data[i + 4:i + 4 + n])
    assert raw == b"\x00" + px[0].tobytes()
