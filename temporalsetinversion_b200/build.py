"""Build recipe for the native library (nvcc, sm_100a, in-tree output).

Compiles temporalsetinversion_b200/csrc/*.cu|*.cpp into
temporalsetinversion_b200/_lib/libtsi.so (loaded by the Python package) and
the same objects into the static library temporalsetinversion_b200/_lib/libtsi.a
(nvcc -lib), which a host program links with the CUDA runtime
(-lcudart_static -lrt -lpthread -ldl, and the C++ runtime).  Device code is built with
--fmad=false so that f32 arithmetic is never contracted into FMA (the
interval formulas and the ray tracer follow the reference's plain f32
operation sequence), host code with -ffp-contract=off for the same reason.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
OBJ_DIR = ROOT / "_build" / "obj"
LIB = OUT_DIR / "libtsi.so"
STATIC_LIB = OUT_DIR / "libtsi.a"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    "-I", str(ROOT / "include"), "-I", str(CSRC),
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cc_flags() -> list:
    # the system compiler; an alternative toolchain on PATH may lack pieces nvcc expects
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def sources() -> list:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _deps_newer(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    if src.stat().st_mtime > t:
        return True
    for h in list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "tsi.h"]:
        if h.stat().st_mtime > t:
            return True
    return False


def build(verbose: bool = False, force: bool = False) -> Path:
    nvcc = _nvcc()
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    jobs = []
    for src in sources():
        obj = OBJ_DIR / (src.name + ".o")
        if force or _deps_newer(obj, src):
            jobs.append([nvcc] + _host_cc_flags() + NVFLAGS + ["-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda cmd: subprocess.run(cmd, capture_output=True, text=True), jobs))
    for cmd, r in zip(jobs, results):
        if verbose or r.returncode:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError("nvcc failed on %s" % cmd[-3])
    objs = [str(OBJ_DIR / (s.name + ".o")) for s in sources()]
    if force or jobs or not LIB.exists():
        cmd = [nvcc] + _host_cc_flags() + ARCH + ["-shared", "-o", str(LIB)] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            raise RuntimeError("link failed")
    if force or jobs or not STATIC_LIB.exists():
        if STATIC_LIB.exists():
            STATIC_LIB.unlink()
        cmd = [nvcc] + _host_cc_flags() + ARCH + ["-lib", "-o", str(STATIC_LIB)] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            raise RuntimeError("static library failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
