"""TEST INFRASTRUCTURE: Python access to the CPU oracle (oracle/tsi_oracle.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this package, as the checker or the timed CPU reference.  The product
(temporalsetinversion_b200) never imports it.

Parity status: unpinned against the reference's own outputs (the reference
is WGSL under wgpu/Vulkan and cannot run on these machines; it has no tests
or golden vectors).  The oracle restates compute.wgsl and ir.rs line by line
(see the header of tsi_oracle.cpp) and is pinned to the reference's scene
fixtures only through the tape lowering (tests/golden/tapes).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libtsi_oracle.so"

CELL_DTYPE = np.dtype([
    ("level", "<u4"), ("ix", "<u4"), ("iy", "<u4"), ("iz", "<u4"), ("f", "<f4"), ("t", "<f4"),
    ("time_err", "<f4"), ("fast", "<f4"), ("dx", "<f4"), ("dy", "<f4"), ("dz", "<f4"), ("has_children", "<u4"),
    ("x", "<f4", 2), ("y", "<f4", 2), ("z", "<f4", 2),
])

STATS_FIELDS = ["parents_expanded", "cells_evaluated", "cells_reverse", "cells_skipped", "cells_ambiguous",
                "cells_empty", "cells_full", "cells_enqueued", "cells_reused", "instr_forward", "instr_reverse"]


class _Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in STATS_FIELDS] + [("levels", C.c_uint32), ("pad", C.c_uint32)]


_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (outputs under oracle/_build)."""
    r = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        src_t = max((HERE / f).stat().st_mtime for f in ("tsi_oracle.cpp", "oracle_fmath.h", "Makefile"))
        if not LIB.exists() or LIB.stat().st_mtime < src_t:
            build()
        lib = C.CDLL(str(LIB))
        vp, u32, u64, f32, fp = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float, C.POINTER(C.c_float)
        lib.oracle_eval_boxes.argtypes = [vp, u32, u32, fp, C.c_int, fp]
        lib.oracle_scene_create.restype = vp
        lib.oracle_scene_create.argtypes = [vp, u32, vp]
        lib.oracle_scene_destroy.argtypes = [vp]
        lib.oracle_scene_reset.argtypes = [vp]
        lib.oracle_scene_invert.argtypes = [vp, f32, f32, vp]
        lib.oracle_scene_cells.restype = u64
        lib.oracle_scene_cells.argtypes = [vp, vp, u64]
        lib.oracle_scene_voxels_live.restype = u64
        lib.oracle_scene_voxels_live.argtypes = [vp]
        lib.oracle_scene_trace.argtypes = [vp, vp, fp, fp, fp, u32, u32, C.POINTER(u64)]
        for name in ("oracle_sin", "oracle_exp", "oracle_log", "oracle_cos", "oracle_acos", "oracle_linear_to_srgb"):
            getattr(lib, name).restype = f32
            getattr(lib, name).argtypes = [f32]
        for name in ("oracle_atan2", "oracle_fmin", "oracle_fmax"):
            getattr(lib, name).restype = f32
            getattr(lib, name).argtypes = [f32, f32]
        lib.oracle_frand_seq.argtypes = [u32, u32, fp]
        lib.oracle_sunsky.argtypes = [fp, f32, f32, fp]
        lib.oracle_powi.restype = f32
        lib.oracle_powi.argtypes = [f32, C.c_int]
        lib.oracle_num_threads.restype = C.c_int
        lib.oracle_set_threads.argtypes = [C.c_int]
        _lib = lib
    return _lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def eval_boxes(gpu_instructions: np.ndarray, boxes: np.ndarray, reverse: bool = True) -> np.ndarray:
    lib = load()
    tape = np.ascontiguousarray(gpu_instructions)
    boxes = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 8)
    out = np.zeros((len(boxes), 10), dtype=np.float32)
    rc = lib.oracle_eval_boxes(tape.ctypes.data, len(tape), len(boxes), _fp(boxes), int(reverse), _fp(out))
    assert rc == 0
    return out


class Scene:
    """CPU restatement of one scene's resident octree."""

    def __init__(self, gpu_instructions: np.ndarray, params):
        self.lib = load()
        self._tape = np.ascontiguousarray(gpu_instructions)
        self._params = params  # a ctypes struct with tsi_params' layout
        self.h = self.lib.oracle_scene_create(self._tape.ctypes.data, len(self._tape), C.addressof(params))

    def reset(self):
        self.lib.oracle_scene_reset(self.h)

    def invert(self, time: float, t0: float = math.nan) -> dict:
        st = _Stats()
        self.lib.oracle_scene_invert(self.h, float(time), float(t0), C.byref(st))
        d = {n: getattr(st, n) for n in STATS_FIELDS}
        d["levels"] = st.levels
        return d

    def cells(self) -> np.ndarray:
        n = self.lib.oracle_scene_cells(self.h, None, 0)
        arr = np.zeros(n, dtype=CELL_DTYPE)
        self.lib.oracle_scene_cells(self.h, arr.ctypes.data, n)
        return arr

    def voxels_live(self) -> int:
        return int(self.lib.oracle_scene_voxels_live(self.h))

    def trace(self, uniforms, rows=None) -> dict:
        w, h = uniforms.resolution[0], uniforms.resolution[1]
        y0, y1 = (0, h) if rows is None else rows
        rgba = np.zeros((h, w, 4), dtype=np.float32)
        depth = np.full((h, w), np.nan, dtype=np.float32)
        normal = np.zeros((h, w, 3), dtype=np.float32)
        visits = C.c_uint64(0)
        self.lib.oracle_scene_trace(self.h, C.addressof(uniforms), _fp(rgba), _fp(depth), _fp(normal), y0, y1,
                                    C.byref(visits))
        return {"rgba": rgba, "depth": depth, "normal": normal, "visits": visits.value}

    def __del__(self):
        try:
            self.lib.oracle_scene_destroy(self.h)
        except Exception:
            pass


def frand_seq(seed: int, n: int) -> np.ndarray:
    """frand, frand0to1, frand, ... (compute.wgsl:2451-2472) from one seed."""
    lib = load()
    out = np.zeros(n, np.float32)
    lib.oracle_frand_seq(C.c_uint32(seed), C.c_uint32(n), _fp(out))
    return out


def sunsky(view, sun) -> np.ndarray:
    lib = load()
    v = np.asarray(view, np.float32)
    out = np.zeros(3, np.float32)
    lib.oracle_sunsky(_fp(v), C.c_float(sun[0]), C.c_float(sun[1]), _fp(out))
    return out


def set_threads(n: int) -> None:
    load().oracle_set_threads(int(n))


def num_threads() -> int:
    return int(load().oracle_num_threads())
