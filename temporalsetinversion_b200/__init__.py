"""B200-native temporal set inversion (interval octree inversion of animated
implicits, temporal error bound, per-cell tape pruning, octree ray tracing).

The compute path is libtsi.so (CUDA, sm_100a) behind the C ABI of
include/tsi.h; this package is its Python host.
"""
from .api import CELL_DTYPE, IR, Device, Scene, Server, State, Tape, default_params, make_uniforms  # noqa: F401
from . import scenes  # noqa: F401

__all__ = ["IR", "Device", "Tape", "Scene", "Server", "State", "default_params", "make_uniforms", "scenes",
           "CELL_DTYPE"]
