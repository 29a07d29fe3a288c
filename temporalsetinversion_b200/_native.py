"""ctypes binding of the C ABI in include/tsi.h (libtsi.so, built in-tree).

The library is the product; this module only declares its structs and entry
points.  Loading fails loudly when the shared object is missing: there is no
Python or CPU fallback for any compute entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "_lib" / "libtsi.so"

u32, i32, u64, f32 = C.c_uint32, C.c_int32, C.c_uint64, C.c_float
P = C.POINTER

TSI_OK = 0
STATUS_NAMES = {
    0: "TSI_OK", 1: "TSI_ERR_INVALID_ARGUMENT", 2: "TSI_ERR_PARSE", 3: "TSI_ERR_CUDA", 4: "TSI_ERR_OOM",
    5: "TSI_ERR_QUEUE_FULL", 6: "TSI_ERR_WATCHDOG", 7: "TSI_ERR_BAD_OPCODE", 8: "TSI_ERR_TAPE_TOO_WIDE",
    9: "TSI_ERR_NO_DEVICE", 10: "TSI_ERR_BUFFER_TOO_SMALL", 11: "TSI_ERR_BUSY", 12: "TSI_ERR_NOT_FOUND",
    13: "TSI_ERR_SHUTDOWN",
}


class GPUInstruction(C.Structure):  # ir.rs:88-97
    _fields_ = [("index_", u32), ("opcode_uses", u32), ("larg_rarg", u32), ("literal", f32),
                ("val", f32 * 2), ("sens", f32 * 2)]


class Params(C.Structure):
    _fields_ = [("localsubdiv", i32), ("delta", f32), ("pointsample", i32), ("fastenabled", i32),
                ("lipschitz_corrected", i32), ("swept_volume", i32), ("fast_normals", i32), ("normal_viz", i32),
                ("rounding_mode", i32), ("fast_multiplier", f32), ("scene_id", i32),
                ("octree_darken_factor", f32), ("root_lo", f32 * 3), ("root_hi", f32 * 3), ("pruning", i32),
                ("swept_dt", f32), ("cinematic", i32), ("samples", i32), ("see_background", i32)]


class Uniforms(C.Structure):  # uniforms.rs:8-17
    _fields_ = [("view_matrix", f32 * 16), ("resolution", u32 * 2), ("time", f32), ("lasttime", f32),
                ("rendermode", f32), ("_padding", f32 * 3)]


LEVEL_COUNTERS = ["parents", "evaluated", "reverse", "skipped", "ambiguous", "empty", "full", "enqueued", "reused",
                  "instr_fwd", "instr_rev", "instr_full", "fp32", "brick_alloc", "brick_free", "tape_words",
                  "prune_fallback", "wide_items", "cyc_wide", "cyc_wide_max", "cyc_wide_fwd", "cyc_wide_rev",
                  "cyc_narrow", "cyc_narrow_max", "narrow_long", "narrow_len_max",
                  "cyc_n_fwd", "cyc_n_rev", "cyc_n_prune", "n_fwd_instr",
                  "wide_fin", "cyc_fin_live", "cyc_fin_compact", "cyc_fin_push", "wide_refwd", "cyc_wide_refwd"]


class Stats(C.Structure):
    _fields_ = [(n, u64) for n in (
        "parents_expanded", "cells_evaluated", "cells_reverse", "cells_skipped", "cells_ambiguous", "cells_empty",
        "cells_full", "cells_enqueued", "cells_reused", "instr_forward", "instr_reverse", "instr_full_equiv",
        "fp32_ops", "bricks_allocated", "bricks_freed", "voxels_live", "items_high_water", "tape_words",
        "prune_fallbacks", "fp32_ops_full_fwd", "fp32_ops_full_rev", "cells_unpruned_regs")] + [("levels", u32), ("error_flags", u32), ("device_ms", f32), ("reserved", f32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Cell(C.Structure):
    _fields_ = [("level", u32), ("ix", u32), ("iy", u32), ("iz", u32), ("f", f32), ("t", f32), ("time_err", f32),
                ("fast", f32), ("dx", f32), ("dy", f32), ("dz", f32), ("has_children", u32), ("x", f32 * 2),
                ("y", f32 * 2), ("z", f32 * 2)]


AUTOTUNE_MAX = 16


class AutotuneResult(C.Structure):
    _fields_ = [("wide_threshold", u32), ("candidates", u32), ("threshold", u32 * AUTOTUNE_MAX),
                ("ms", f32 * AUTOTUNE_MAX), ("deep_level", u32), ("deep_threshold", u32),
                ("narrow_parents", u32), ("wide_prune_level", u32)]


SERVER_STATIC_BATCHES = 1


class ServerOpts(C.Structure):
    _fields_ = [("max_batch", u32), ("flags", u32), ("max_queue", u32), ("reserved", u32)]


class ServerStats(C.Structure):
    _fields_ = [("completed", u64), ("batches", u64), ("mean_batch", f32), ("p50_ms", f32), ("p99_ms", f32),
                ("max_ms", f32), ("queued", u32)]


class Image(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("rgba", P(f32)), ("depth", P(f32)), ("normal", P(f32))]


class ImageDevice(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("rgba", C.c_void_p), ("depth", C.c_void_p),
                ("normal", C.c_void_p)]


class FrameDevice(C.Structure):  # tsi_frame_device: caller-owned device buffers of a composited frame
    _fields_ = [("width", u32), ("height", u32), ("rgba", C.c_void_p), ("depth", C.c_void_p),
                ("normal", C.c_void_p), ("key", C.c_void_p)]


class DeviceOpts(C.Structure):
    _fields_ = [("device", i32), ("work_item_capacity", u64), ("tape_arena_words", u64), ("log_arena_bytes", u64),
                ("watchdog_iters", u32), ("max_scenes_per_launch", u32), ("wide_smem_bytes", u32),
                ("hbm_budget_bytes", u64)]


class TapeInfo(C.Structure):
    _fields_ = [("instruction_count", u32), ("registers", u32), ("minmax_count", u32), ("reserved", u32)]


class Request(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("time", f32), ("t0_or_nan", f32), ("uniforms", P(Uniforms)),
                ("out", P(Image)), ("stats", P(Stats))]


# every symbol declared in include/tsi.h, with its signature
SIGNATURES = {
    "tsi_version": (u32, []),
    "tsi_status_string": (C.c_char_p, [i32]),
    "tsi_default_params": (None, [P(Params)]),
    "tsi_create": (i32, [P(DeviceOpts), P(C.c_void_p)]),
    "tsi_destroy": (None, [C.c_void_p]),
    "tsi_synchronize": (i32, [C.c_void_p]),
    "tsi_ir_lower": (i32, [C.c_char_p, C.c_size_t, f32, P(GPUInstruction), u32, P(u32)]),
    "tsi_tape_upload": (i32, [C.c_void_p, P(GPUInstruction), u32, P(C.c_void_p)]),
    "tsi_tape_from_llvm_ir": (i32, [C.c_void_p, C.c_char_p, C.c_size_t, P(C.c_void_p)]),
    "tsi_tape_info_get": (i32, [C.c_void_p, P(TapeInfo)]),
    "tsi_tape_destroy": (None, [C.c_void_p]),
    "tsi_tape_eval_boxes": (i32, [C.c_void_p, C.c_void_p, u32, P(f32), i32, i32, P(f32)]),
    "tsi_scene_create": (i32, [C.c_void_p, C.c_void_p, P(Params), u64, P(C.c_void_p)]),
    "tsi_scene_destroy": (None, [C.c_void_p]),
    "tsi_scene_reset": (i32, [C.c_void_p]),
    "tsi_scene_invert": (i32, [C.c_void_p, f32, f32, P(Stats)]),
    "tsi_scene_trace": (i32, [C.c_void_p, P(Uniforms), P(Image), P(Stats)]),
    "tsi_scene_image_device": (i32, [C.c_void_p, P(ImageDevice)]),
    "tsi_scene_readback_cells": (i32, [C.c_void_p, P(Cell), u64, P(u64)]),
    "tsi_scene_readback_leaves": (i32, [C.c_void_p, P(u32), u64, P(u64)]),
    "tsi_scene_snapshot_size": (i32, [C.c_void_p, P(u64)]),
    "tsi_scene_snapshot": (i32, [C.c_void_p, C.c_void_p, u64, P(u64)]),
    "tsi_scene_restore": (i32, [C.c_void_p, C.c_void_p, u64]),
    "tsi_scene_get_params": (i32, [C.c_void_p, P(Params)]),
    "tsi_scene_device_bytes": (u64, [C.c_void_p]),
    "tsi_batch_run": (i32, [C.c_void_p, P(Request), u32]),
    "tsi_server_create": (i32, [C.c_void_p, P(ServerOpts), P(C.c_void_p)]),
    "tsi_server_submit": (i32, [C.c_void_p, P(Request), P(u64)]),
    "tsi_server_poll": (i32, [C.c_void_p, u64, u32, P(f32)]),
    "tsi_server_stats_get": (i32, [C.c_void_p, P(ServerStats)]),
    "tsi_server_destroy": (None, [C.c_void_p]),
    "tsi_batch_graph_create": (i32, [C.c_void_p, P(Request), u32, P(C.c_void_p)]),
    "tsi_scene_image_copy": (i32, [C.c_void_p, P(Image)]),
    "tsi_scene_trace_async": (i32, [C.c_void_p, P(Uniforms), P(Image)]),
    "tsi_scene_invert_async": (i32, [C.c_void_p, f32, f32]),
    "tsi_rgba8_from_frame": (None, [P(f32), u64, P(C.c_uint8)]),
    "tsi_scenes_device_bytes": (u64, [C.c_void_p]),
    "tsi_scene_invert_wait": (i32, [C.c_void_p, P(Stats)]),
    "tsi_scene_trace_wait": (i32, [C.c_void_p]),
    "tsi_batch_graph_launch": (i32, [C.c_void_p]),
    "tsi_batch_graph_wait": (i32, [C.c_void_p, P(Stats)]),
    "tsi_batch_autotune": (i32, [C.c_void_p, P(Request), u32, u32, P(AutotuneResult)]),
    "tsi_tape_wide_threshold": (u32, [C.c_void_p]),
    "tsi_tape_set_wide_threshold": (i32, [C.c_void_p, u32]),
    "tsi_tape_set_wide_threshold_deep": (i32, [C.c_void_p, u32, u32]),
    "tsi_tape_wide_threshold_deep": (i32, [C.c_void_p, C.POINTER(u32), C.POINTER(u32)]),
    "tsi_tape_set_narrow_parents": (i32, [C.c_void_p, u32]),
    "tsi_tape_narrow_parents": (u32, [C.c_void_p]),
    "tsi_tape_set_wide_prune_level": (i32, [C.c_void_p, u32]),
    "tsi_tape_wide_prune_level": (u32, [C.c_void_p]),
    "tsi_scene_autotune": (i32, [C.c_void_p, P(f32), u32, u32, P(AutotuneResult)]),
    "tsi_batch_graph_destroy": (None, [C.c_void_p]),
    "tsi_last_error": (C.c_char_p, []),
    "tsi_ir_tape_info": (i32, [C.c_char_p, C.c_size_t, P(TapeInfo), P(u32), u32]),
    "tsi_compile_gpu_instructions": (i32, [P(GPUInstruction), u32, P(u32), u32, P(TapeInfo)]),
    "tsi_debug_math": (i32, [C.c_void_p, i32, u32, P(f32), P(f32), P(f32)]),
    "tsi_debug_level_profile": (i32, [C.c_void_p, u32, P(f32), P(u64), P(u32)]),
    "tsi_compile_wide_gpu_instructions": (i32, [P(GPUInstruction), u32, P(u32), u32, P(u32), u32, P(TapeInfo),
                                                 P(u32)]),
    "tsi_tape_eval_boxes_static": (i32, [C.c_void_p, u32, C.c_void_p, i32, i32, C.c_void_p, C.c_void_p]),
    "tsi_static_scratch_bytes": (u64, []),
    "tsi_params_subtree": (i32, [P(Params), u32, u32, P(Params)]),
    "tsi_frames_composite": (i32, [C.c_void_p, P(C.c_void_p), P(u32), u32, P(FrameDevice)]),
    "tsi_frame_keep_nearest": (i32, [C.c_void_p, C.c_void_p, P(FrameDevice)]),
}

_lib = None


def load() -> C.CDLL:
    """Load libtsi.so (building it first if a toolchain is available)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        if os.environ.get("TSI_NO_BUILD"):
            raise RuntimeError("libtsi.so is missing at %s (build it with temporalsetinversion_b200/build.py)" % LIB_PATH)
        from . import build as _build
        _build.build()
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class TsiError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = load()
        detail = lib.tsi_last_error().decode(errors="replace")
        super().__init__("%s failed: %s (%s)%s" % (where, STATUS_NAMES.get(status, status),
                                                   lib.tsi_status_string(status).decode(),
                                                   (": " + detail) if detail else ""))
        self.status = status


def check(status: int, where: str) -> None:
    if status != TSI_OK:
        raise TsiError(status, where)
