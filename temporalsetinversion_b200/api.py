"""Python host over the C ABI, mirroring the reference's host interface.

The reference host (Rust) lowers the scene (`ir::IR::new`, src/ir.rs:334),
seeds and dispatches `main` once per frame (`State::compute`,
src/main.rs:724-820) and dispatches `rt_main` (`State::render`,
main.rs:639-656) with the uniforms of src/uniforms.rs.  The same steps here
go through libtsi.so:

    ir = IR.new(text, time)                 # ir.rs IR::new
    dev = Device()                          # State::new's device setup
    state = State(dev, text, params)        # + tapes[0] upload, first_eval
    ms = state.compute(time)                # State::compute -> device ms
    img = state.render(uniforms)            # State::render (headless)
"""
from __future__ import annotations

import ctypes as C
import math
import weakref
from dataclasses import dataclass

import numpy as np

from . import _native as N

__all__ = ["IR", "Device", "Tape", "Scene", "State", "default_params", "make_uniforms", "CELL_DTYPE"]

CELL_DTYPE = np.dtype([
    ("level", "<u4"), ("ix", "<u4"), ("iy", "<u4"), ("iz", "<u4"), ("f", "<f4"), ("t", "<f4"),
    ("time_err", "<f4"), ("fast", "<f4"), ("dx", "<f4"), ("dy", "<f4"), ("dz", "<f4"), ("has_children", "<u4"),
    ("x", "<f4", 2), ("y", "<f4", 2), ("z", "<f4", 2),
])
GPU_INSTR_DTYPE = np.dtype([("index_", "<u4"), ("opcode_uses", "<u4"), ("larg_rarg", "<u4"), ("literal", "<f4"),
                            ("val", "<f4", 2), ("sens", "<f4", 2)])
assert CELL_DTYPE.itemsize == C.sizeof(N.Cell)
assert GPU_INSTR_DTYPE.itemsize == C.sizeof(N.GPUInstruction)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def default_params(**kw) -> N.Params:
    """PARAMETERS block defaults (compute.wgsl:3494-3511), overridable by name."""
    lib = N.load()
    p = N.Params()
    lib.tsi_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        if k in ("root_lo", "root_hi"):
            for i in range(3):
                getattr(p, k)[i] = float(v[i])
        else:
            setattr(p, k, v)
    return p


def make_uniforms(view, resolution, time: float = 0.0, lasttime: float = 0.0, rendermode: float = 0.0) -> N.Uniforms:
    """uniforms.rs:8-45: camera-to-world view matrix (16 floats, column
    major), resolution, time."""
    u = N.Uniforms()
    for i, v in enumerate(view):
        u.view_matrix[i] = float(v)
    u.resolution[0], u.resolution[1] = int(resolution[0]), int(resolution[1])
    u.time = float(time)
    u.lasttime = float(lasttime)
    u.rendermode = float(rendermode)
    return u


class IR:
    """ir.rs `IR`: `instructions` in the 32-byte GPUInstruction layout."""

    def __init__(self, gpu_instructions: np.ndarray):
        self.gpu_instructions = gpu_instructions

    @classmethod
    def new(cls, text: str, time: float = 0.0) -> "IR":
        lib = N.load()
        raw = text.encode()
        n = C.c_uint32(0)
        N.check(lib.tsi_ir_lower(raw, len(raw), float(time), None, 0, C.byref(n)), "tsi_ir_lower")
        arr = np.zeros(n.value, dtype=GPU_INSTR_DTYPE)
        N.check(lib.tsi_ir_lower(raw, len(raw), float(time), arr.ctypes.data_as(C.POINTER(N.GPUInstruction)),
                                 n.value, C.byref(n)), "tsi_ir_lower")
        return cls(arr)

    def __len__(self) -> int:
        return len(self.gpu_instructions)


class Device:
    """A tsi_ctx on one CUDA device (fails with TSI_ERR_NO_DEVICE without one)."""

    def __init__(self, device: int = 0, work_item_capacity: int = 0, tape_arena_words: int = 0,
                 log_arena_bytes: int = 0, max_scenes_per_launch: int = 0, wide_smem_bytes: int = 0,
                 hbm_budget_bytes: int = 0):
        self.lib = N.load()
        opts = N.DeviceOpts(device, work_item_capacity, tape_arena_words, log_arena_bytes, 0, max_scenes_per_launch,
                            wide_smem_bytes, hbm_budget_bytes)
        h = C.c_void_p()
        N.check(self.lib.tsi_create(C.byref(opts), C.byref(h)), "tsi_create")
        self.handle = h
        self.index = int(device)  # CUDA ordinal
        self._children = weakref.WeakSet()

    def close(self) -> None:
        if getattr(self, "handle", None):
            for child in list(self._children):  # scenes first, then tapes
                if isinstance(child, Scene):
                    child.close()
            for child in list(self._children):
                child.close()
            self.lib.tsi_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def scenes_bytes(self) -> int:
        """Device bytes the scenes of this device hold (tsi_scenes_device_bytes)."""
        return int(self.lib.tsi_scenes_device_bytes(self.handle))

    def synchronize(self) -> None:
        N.check(self.lib.tsi_synchronize(self.handle), "tsi_synchronize")

    def level_profile(self, max_levels: int = 24) -> list:
        """Per-level ms and counters of the last inversion on this device."""
        ms = np.zeros(max_levels, np.float32)
        cnt = np.zeros((max_levels, len(N.LEVEL_COUNTERS)), np.uint64)
        n = C.c_uint32(0)
        N.check(self.lib.tsi_debug_level_profile(self.handle, max_levels, _fptr(ms),
                                                 cnt.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(n)),
                "tsi_debug_level_profile")
        return [dict(level=l, ms=float(ms[l]), **{k: int(cnt[l, i]) for i, k in enumerate(N.LEVEL_COUNTERS)})
                for l in range(min(n.value, max_levels))]

    def math(self, which: int, a: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.float32)
        b = np.zeros_like(a) if b is None else np.ascontiguousarray(b, dtype=np.float32)
        out = np.empty_like(a)
        N.check(self.lib.tsi_debug_math(self.handle, which, a.size, _fptr(a), _fptr(b), _fptr(out)), "tsi_debug_math")
        return out


class Tape:
    def __init__(self, device: Device, handle: C.c_void_p):
        self.device = device
        self.handle = handle
        device._children.add(self)
        info = N.TapeInfo()
        N.check(device.lib.tsi_tape_info_get(handle, C.byref(info)), "tsi_tape_info_get")
        self.instruction_count = info.instruction_count
        self.registers = info.registers
        self.minmax_count = info.minmax_count

    @classmethod
    def from_llvm_ir(cls, device: Device, text: str) -> "Tape":
        raw = text.encode()
        h = C.c_void_p()
        N.check(device.lib.tsi_tape_from_llvm_ir(device.handle, raw, len(raw), C.byref(h)), "tsi_tape_from_llvm_ir")
        return cls(device, h)

    @classmethod
    def upload(cls, device: Device, gpu_instructions: np.ndarray) -> "Tape":
        arr = np.ascontiguousarray(gpu_instructions, dtype=GPU_INSTR_DTYPE)
        h = C.c_void_p()
        N.check(device.lib.tsi_tape_upload(device.handle, arr.ctypes.data_as(C.POINTER(N.GPUInstruction)), len(arr),
                                           C.byref(h)), "tsi_tape_upload")
        return cls(device, h)

    def eval_boxes(self, boxes: np.ndarray, rounding_mode: int = 0, reverse: bool = True) -> np.ndarray:
        boxes = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 8)
        out = np.zeros((len(boxes), 10), dtype=np.float32)
        N.check(self.device.lib.tsi_tape_eval_boxes(self.device.handle, self.handle, len(boxes), _fptr(boxes),
                                                    rounding_mode, int(reverse), _fptr(out)), "tsi_tape_eval_boxes")
        return out

    @property
    def wide_threshold(self) -> int:
        """Pruned-tape length from which child cells take the wide path
        (0xffffffff: narrow only)."""
        return int(self.device.lib.tsi_tape_wide_threshold(self.handle))

    @wide_threshold.setter
    def wide_threshold(self, v: int) -> None:
        N.check(self.device.lib.tsi_tape_set_wide_threshold(self.handle, int(v)), "tsi_tape_set_wide_threshold")

    @property
    def wide_threshold_deep(self) -> tuple:
        """(level, threshold): child cells at that octree level or deeper use
        the second threshold (level 0xffffffff: off)."""
        lv, th = C.c_uint32(0), C.c_uint32(0)
        N.check(self.device.lib.tsi_tape_wide_threshold_deep(self.handle, C.byref(lv), C.byref(th)),
                "tsi_tape_wide_threshold_deep")
        return int(lv.value), int(th.value)

    @wide_threshold_deep.setter
    def wide_threshold_deep(self, v: tuple) -> None:
        N.check(self.device.lib.tsi_tape_set_wide_threshold_deep(self.handle, int(v[0]), int(v[1])),
                "tsi_tape_set_wide_threshold_deep")

    @property
    def narrow_parents(self) -> int:
        """Parents per narrow work item above the leaf level (1, 2 or 4)."""
        return int(self.device.lib.tsi_tape_narrow_parents(self.handle))

    @narrow_parents.setter
    def narrow_parents(self, v: int) -> None:
        N.check(self.device.lib.tsi_tape_set_narrow_parents(self.handle, int(v)), "tsi_tape_set_narrow_parents")

    @property
    def wide_prune_level(self) -> int:
        """First parent level whose wide groups prune the tape for their
        children (0xffffffff: half the scene's levels)."""
        return int(self.device.lib.tsi_tape_wide_prune_level(self.handle))

    @wide_prune_level.setter
    def wide_prune_level(self, v: int) -> None:
        N.check(self.device.lib.tsi_tape_set_wide_prune_level(self.handle, int(v)), "tsi_tape_set_wide_prune_level")

    def close(self) -> None:
        if getattr(self, "handle", None) and getattr(self.device, "handle", None):
            self.device.lib.tsi_tape_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """Resident octree of one scene (tsi_scene)."""

    def __init__(self, device: Device, tape: Tape, params: N.Params, voxel_capacity: int = 0):
        self.device, self.tape, self.params = device, tape, params
        h = C.c_void_p()
        N.check(device.lib.tsi_scene_create(device.handle, tape.handle, C.byref(params), voxel_capacity, C.byref(h)),
                "tsi_scene_create")
        self.handle = h
        device._children.add(self)

    def reset(self) -> None:
        N.check(self.device.lib.tsi_scene_reset(self.handle), "tsi_scene_reset")

    def autotune(self, times: list, reps: int = 2) -> dict:
        """Picks the tape's wide threshold, then a deep-level one, then the
        parents per narrow item, then the wide path's prune level, by timing
        inversions over `times` (tsi_scene_autotune); the scene is left
        reset."""
        arr = (C.c_float * len(times))(*[float(t) for t in times])
        r = N.AutotuneResult()
        N.check(self.device.lib.tsi_scene_autotune(self.handle, arr, len(times), int(reps), C.byref(r)),
                "tsi_scene_autotune")
        return {"wide_threshold": int(r.wide_threshold), "deep_level": int(r.deep_level),
                "deep_threshold": int(r.deep_threshold), "narrow_parents": int(r.narrow_parents),
                "wide_prune_level": int(r.wide_prune_level),
                "trials": [(int(r.threshold[k]), float(r.ms[k])) for k in range(r.candidates)]}

    def invert(self, time: float, t0: float = math.nan) -> N.Stats:
        st = N.Stats()
        N.check(self.device.lib.tsi_scene_invert(self.handle, float(time), float(t0), C.byref(st)), "tsi_scene_invert")
        return st

    def invert_async(self, time: float, t0: float = math.nan) -> None:
        """tsi_scene_invert_async: queue the frame's inversion and return."""
        N.check(self.device.lib.tsi_scene_invert_async(self.handle, float(time), float(t0)), "tsi_scene_invert_async")

    def invert_wait(self) -> N.Stats:
        """tsi_scene_invert_wait: wait for the queued inversions; raises on a
        device error in any of them; counters of the last one."""
        st = N.Stats()
        N.check(self.device.lib.tsi_scene_invert_wait(self.handle, C.byref(st)), "tsi_scene_invert_wait")
        return st

    def trace(self, uniforms: N.Uniforms, rgba: bool = True, depth: bool = True, normal: bool = True) -> dict:
        w, h = uniforms.resolution[0], uniforms.resolution[1]
        out = {}
        img = N.Image(w, h, None, None, None)
        if rgba:
            out["rgba"] = np.empty((h, w, 4), dtype=np.float32)
            img.rgba = _fptr(out["rgba"])
        if depth:
            out["depth"] = np.empty((h, w), dtype=np.float32)
            img.depth = _fptr(out["depth"])
        if normal:
            out["normal"] = np.empty((h, w, 3), dtype=np.float32)
            img.normal = _fptr(out["normal"])
        st = N.Stats()
        N.check(self.device.lib.tsi_scene_trace(self.handle, C.byref(uniforms), C.byref(img), C.byref(st)),
                "tsi_scene_trace")
        out["device_ms"] = st.device_ms
        out["visits"] = st.reserved
        return out

    def trace_async(self, uniforms: N.Uniforms, rgba, depth=None, normal=None) -> None:
        """tsi_scene_trace_async: queue the trace and the frame's copy into
        the given host arrays (float32, C-contiguous; pinned memory, e.g. a
        pinned torch tensor's numpy view, makes the copy asynchronous).  The
        arrays must stay untouched until trace_wait()."""
        w, h = uniforms.resolution[0], uniforms.resolution[1]
        img = N.Image(w, h, None, None, None)
        keep = []
        for name, arr, n in (("rgba", rgba, 4), ("depth", depth, 1), ("normal", normal, 3)):
            if arr is None:
                continue
            if arr.dtype != np.float32 or not arr.flags.c_contiguous or arr.size != w * h * n:
                raise ValueError("%s must be a C-contiguous float32 array of %d values" % (name, w * h * n))
            setattr(img, name, _fptr(arr))
            keep.append(arr)
        N.check(self.device.lib.tsi_scene_trace_async(self.handle, C.byref(uniforms), C.byref(img)),
                "tsi_scene_trace_async")
        self._async_keep = (keep, uniforms)

    def trace_wait(self) -> None:
        N.check(self.device.lib.tsi_scene_trace_wait(self.handle), "tsi_scene_trace_wait")
        self._async_keep = None

    def cells(self) -> np.ndarray:
        lib = self.device.lib
        n = C.c_uint64(0)
        N.check(lib.tsi_scene_readback_cells(self.handle, None, 0, C.byref(n)), "tsi_scene_readback_cells")
        arr = np.zeros(n.value, dtype=CELL_DTYPE)
        N.check(lib.tsi_scene_readback_cells(self.handle, arr.ctypes.data_as(C.POINTER(N.Cell)), n.value,
                                             C.byref(n)), "tsi_scene_readback_cells")
        return arr

    def image(self, width: int, height: int) -> dict:
        """The last rendered frame (kept on the device by graph replays and
        the server) copied to host arrays."""
        out = {"rgba": np.empty((height, width, 4), np.float32), "depth": np.empty((height, width), np.float32),
               "normal": np.empty((height, width, 3), np.float32)}
        img = N.Image(width, height, _fptr(out["rgba"]), _fptr(out["depth"]), _fptr(out["normal"]))
        N.check(self.device.lib.tsi_scene_image_copy(self.handle, C.byref(img)), "tsi_scene_image_copy")
        return out

    def device_bytes(self) -> int:
        """Device bytes of this scene's pool and frame buffers."""
        return int(self.device.lib.tsi_scene_device_bytes(self.handle))

    def snapshot(self) -> bytes:
        """The resident octree as a host blob (tsi_scene_snapshot)."""
        lib = self.device.lib
        n = C.c_uint64(0)
        N.check(lib.tsi_scene_snapshot_size(self.handle, C.byref(n)), "tsi_scene_snapshot_size")
        buf = C.create_string_buffer(n.value)
        N.check(lib.tsi_scene_snapshot(self.handle, buf, n.value, C.byref(n)), "tsi_scene_snapshot")
        return buf.raw[:n.value]

    def restore(self, blob: bytes) -> None:
        N.check(self.device.lib.tsi_scene_restore(self.handle, blob, len(blob)), "tsi_scene_restore")

    def leaves(self) -> np.ndarray:
        """(level, ix, iy, iz) of the cells the tracer can hit, one row each."""
        lib = self.device.lib
        n = C.c_uint64(0)
        N.check(lib.tsi_scene_readback_leaves(self.handle, None, 0, C.byref(n)), "tsi_scene_readback_leaves")
        arr = np.zeros((n.value, 4), dtype=np.uint32)
        N.check(lib.tsi_scene_readback_leaves(self.handle, arr.ctypes.data_as(C.POINTER(C.c_uint32)), n.value,
                                              C.byref(n)), "tsi_scene_readback_leaves")
        return arr

    def close(self) -> None:
        if getattr(self, "handle", None) and getattr(self.device, "handle", None):
            self.device.lib.tsi_scene_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class FrameResult:
    stats: N.Stats
    rootfind_ms: float


class State:
    """The per-scene state of src/main.rs `State`, headless: compute() is one
    `main` dispatch (with the root re-seeded), render() one `rt_main`."""

    def __init__(self, device: Device, text: str, params: N.Params | None = None, voxel_capacity: int = 0):
        self.device = device
        self.tape = Tape.from_llvm_ir(device, text)
        self.params = params or default_params()
        self.scene = Scene(device, self.tape, self.params, voxel_capacity)
        self.first_eval = False  # the scene is created fresh (main.rs:730)

    def compute(self, time: float, t0: float = math.nan) -> FrameResult:
        if self.first_eval:
            self.scene.reset()
            self.first_eval = False
        st = self.scene.invert(time, t0)
        return FrameResult(st, st.device_ms)

    def render(self, uniforms: N.Uniforms) -> dict:
        return self.scene.trace(uniforms)


def run_batch(device: Device, requests: list, graph: bool = False) -> list:
    """Invert (and trace) several distinct scenes in one fused launch sequence
    (tsi_batch_run).  requests: list of (scene, time, t0, uniforms or None).
    Returns per-request dicts with the frame arrays when uniforms are given."""
    n = len(requests)
    reqs = (N.Request * n)()
    keep = []
    outs = []
    for i, (scene, time, t0, uni) in enumerate(requests):
        reqs[i].scene = scene.handle
        reqs[i].time = float(time)
        reqs[i].t0_or_nan = float(t0)
        st = N.Stats()
        keep.append(st)
        reqs[i].stats = C.pointer(st)
        out = {"stats": st}
        if uni is not None:
            w, h = uni.resolution[0], uni.resolution[1]
            out["rgba"] = np.empty((h, w, 4), np.float32)
            out["depth"] = np.empty((h, w), np.float32)
            out["normal"] = np.empty((h, w, 3), np.float32)
            img = N.Image(w, h, _fptr(out["rgba"]), _fptr(out["depth"]), _fptr(out["normal"]))
            keep += [uni, img]
            reqs[i].uniforms = C.pointer(uni)
            reqs[i].out = C.pointer(img)
        outs.append(out)
    N.check(device.lib.tsi_batch_run(device.handle, reqs, n), "tsi_batch_run")
    return outs


class Server:
    """A worker thread on one device that runs requests with continuous
    batching (tsi_server_*): a request joins the running inversion at the
    next launch step when a slot is free and its scene is idle, and is traced
    on a low-priority stream while the others go on.  With
    static_batches=True it instead fuses the queued requests of distinct
    scenes into one launch sequence at a time.  While it exists, only the
    server uses the device."""

    def __init__(self, device: Device, max_batch: int = 0, static_batches: bool = False, max_queue: int = 0):
        self.device = device
        h = C.c_void_p()
        opts = N.ServerOpts(max_batch, N.SERVER_STATIC_BATCHES if static_batches else 0, max_queue, 0)
        N.check(device.lib.tsi_server_create(device.handle, C.byref(opts), C.byref(h)), "tsi_server_create")
        self.handle = h
        self._keep = {}  # request structs and buffers alive until the ticket completes

    def submit(self, scene: "Scene", time: float, t0: float = float("nan"), uniforms=None,
               image: bool = False) -> int:
        """Queues one request; image=True copies its frame's rgba and depth
        to host arrays that poll() returns."""
        req = N.Request()
        req.scene = scene.handle
        req.time = float(time)
        req.t0_or_nan = float(t0)
        st = N.Stats()
        req.stats = C.pointer(st)
        keep = {"req": req, "stats": st}
        if uniforms is not None:
            keep["uniforms"] = uniforms
            req.uniforms = C.pointer(uniforms)
            if image:
                w, hgt = uniforms.resolution[0], uniforms.resolution[1]
                keep["rgba"] = np.empty((hgt, w, 4), np.float32)
                keep["depth"] = np.empty((hgt, w), np.float32)
                img = N.Image(w, hgt, _fptr(keep["rgba"]), _fptr(keep["depth"]), None)
                keep["img"] = img
                req.out = C.pointer(img)
        ticket = C.c_uint64(0)
        N.check(self.device.lib.tsi_server_submit(self.handle, C.byref(req), C.byref(ticket)), "tsi_server_submit")
        self._keep[ticket.value] = keep
        return ticket.value

    def poll(self, ticket: int, wait_ms: int = 60000, with_depth: bool = False):
        """(stats, latency ms, rgba or None) once done -- with_depth adds the
        depth image -- or None while pending."""
        lat = C.c_float(0.0)
        status = self.device.lib.tsi_server_poll(self.handle, ticket, wait_ms, C.byref(lat))
        if status == 11:  # TSI_ERR_BUSY
            return None
        keep = self._keep.pop(ticket, {})
        N.check(status, "tsi_server_poll")
        if with_depth:
            return keep.get("stats"), lat.value, keep.get("rgba"), keep.get("depth")
        return keep.get("stats"), lat.value, keep.get("rgba")

    def stats(self) -> dict:
        st = N.ServerStats()
        N.check(self.device.lib.tsi_server_stats_get(self.handle, C.byref(st)), "tsi_server_stats_get")
        return {name: getattr(st, name) for name, _ in st._fields_}

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.device.lib.tsi_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def rgba8(rgba: np.ndarray) -> np.ndarray:
    """tsi_rgba8_from_frame: an (H, W, 4) float32 frame as 8-bit RGBA."""
    rgba = np.ascontiguousarray(rgba, dtype=np.float32)
    out = np.empty(rgba.shape, dtype=np.uint8)
    N.load().tsi_rgba8_from_frame(_fptr(rgba), rgba.size // 4, out.ctypes.data_as(C.POINTER(C.c_uint8)))
    return out


def save_png(path, rgba: np.ndarray) -> None:
    """The reference's frame dump (main.rs:692-715): an (H, W, 4) float32
    frame written as an 8-bit RGBA PNG (no compression filters)."""
    import struct
    import zlib

    px = rgba8(rgba)
    h, w = px.shape[0], px.shape[1]
    raw = b"".join(b"\x00" + px[y].tobytes() for y in range(h))

    def chunk(kind: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF)

    png = (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
           chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))
    with open(path, "wb") as f:
        f.write(png)


def batch_autotune(device: Device, requests: list, frames: int = 3) -> dict:
    """tsi_batch_autotune: the wide-threshold multiplier (1, 2, 4 or 8) that
    runs these scenes fastest together.  requests: list of (scene, time).
    The scenes are left reset."""
    n = len(requests)
    reqs = (N.Request * n)()
    for i, (scene, time) in enumerate(requests):
        reqs[i].scene = scene.handle
        reqs[i].time = float(time)
        reqs[i].t0_or_nan = math.nan
    r = N.AutotuneResult()
    N.check(device.lib.tsi_batch_autotune(device.handle, reqs, n, int(frames), C.byref(r)), "tsi_batch_autotune")
    return {"scale": int(r.wide_threshold),
            "trials": [(int(r.threshold[k]), float(r.ms[k])) for k in range(r.candidates)]}


class BatchGraph:
    """tsi_batch_run for a fixed set of distinct scenes captured into a CUDA
    graph; each launch re-reads the requests' times and cameras."""

    def __init__(self, device: Device, requests: list):
        """requests: list of (scene, time, t0, uniforms or None)."""
        self.device = device
        n = len(requests)
        self.reqs = (N.Request * n)()
        self._keep = []
        for i, (scene, time, t0, uni) in enumerate(requests):
            self.reqs[i].scene = scene.handle
            self.reqs[i].time = float(time)
            self.reqs[i].t0_or_nan = float(t0)
            if uni is not None:
                u = N.Uniforms()
                C.memmove(C.byref(u), C.byref(uni), C.sizeof(u))
                self._keep.append(u)
                self.reqs[i].uniforms = C.pointer(u)
            else:
                self._keep.append(None)
        h = C.c_void_p()
        N.check(device.lib.tsi_batch_graph_create(device.handle, self.reqs, n, C.byref(h)), "tsi_batch_graph_create")
        self.handle = h

    def launch(self, times: list, uniforms: list | None = None) -> None:
        for i, t in enumerate(times):
            self.reqs[i].time = float(t)
            if uniforms is not None and uniforms[i] is not None:
                C.memmove(C.byref(self._keep[i]), C.byref(uniforms[i]), C.sizeof(N.Uniforms))
        N.check(self.device.lib.tsi_batch_graph_launch(self.handle), "tsi_batch_graph_launch")

    def wait(self) -> N.Stats:
        """Waits for the last launch; raises on its device error word and
        returns its counters (summed over the batch) and device time."""
        st = N.Stats()
        N.check(self.device.lib.tsi_batch_graph_wait(self.handle, C.byref(st)), "tsi_batch_graph_wait")
        return st

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.device.lib.tsi_batch_graph_destroy(self.handle)
            self.handle = None
