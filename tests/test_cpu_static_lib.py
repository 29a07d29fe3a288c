"""The static library (libtsi.a, nvcc -lib for sm_100a) links into a plain C
host program, the way the reference's Rust host would link it: the program
lowers a scene's LLVM IR through tsi_ir_lower and compares the count with the
shared library's.  No device needed (tsi_create may report no device)."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import pytest

from temporalsetinversion_b200 import api, scenes
from temporalsetinversion_b200 import build as B

ROOT = Path(__file__).resolve().parents[1]

PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include "tsi.h"

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 3;
  fseek(f, 0, SEEK_END);
  long len = ftell(f);
  fseek(f, 0, SEEK_SET);
  char *text = (char *)malloc((size_t)len);
  if (fread(text, 1, (size_t)len, f) != (size_t)len) return 4;
  fclose(f);
  uint32_t n = 0;
  tsi_status st = tsi_ir_lower(text, (size_t)len, 0.0f, NULL, 0, &n);
  if (st != TSI_OK) return 5;
  tsi_gpu_instruction *ins = (tsi_gpu_instruction *)malloc(n * sizeof(tsi_gpu_instruction));
  st = tsi_ir_lower(text, (size_t)len, 0.25f, ins, n, &n);
  if (st != TSI_OK) return 6;
  tsi_ctx *ctx = NULL;
  tsi_status cs = tsi_create(NULL, &ctx);
  if (ctx) tsi_destroy(ctx);
  printf("version %u count %u last_time %.9g opcode_uses %u create %s\n", tsi_version(), n, ins[3].val[0],
         ins[n - 1].opcode_uses, tsi_status_string(cs));
  free(ins);
  free(text);
  return 0;
}
"""


def _cuda_lib_dir() -> Path | None:
    for d in ("/usr/local/cuda/lib64", "/usr/local/cuda/targets/x86_64-linux/lib"):
        if (Path(d) / "libcudart_static.a").exists():
            return Path(d)
    return None


@pytest.mark.skipif(shutil.which("gcc") is None or shutil.which("g++") is None, reason="no host C compiler")
def test_static_library_links_into_a_c_program(tmp_path):
    B.build()
    assert B.STATIC_LIB.exists()
    cuda = _cuda_lib_dir()
    if cuda is None:
        pytest.skip("no libcudart_static.a")
    text = scenes.spheres16(0)
    (tmp_path / "scene.ll").write_text(text)
    (tmp_path / "prog.c").write_text(PROGRAM)
    obj, exe = tmp_path / "prog.o", tmp_path / "prog"
    subprocess.run(["gcc", "-std=c99", "-O1", "-I", str(ROOT / "include"), "-c", str(tmp_path / "prog.c"), "-o",
                    str(obj)], check=True, capture_output=True)
    r = subprocess.run(["g++", str(obj), str(B.STATIC_LIB), "-L", str(cuda), "-lcudart_static", "-lrt", "-lpthread",
                        "-ldl", "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    out = subprocess.run([str(exe), str(tmp_path / "scene.ll")], capture_output=True, text=True, timeout=120,
                         env=dict(os.environ))
    assert out.returncode == 0, out.stderr
    fields = out.stdout.split()
    want = api.IR.new(text, 0.25).gpu_instructions
    assert fields[0] == "version" and int(fields[1]) == 1
    assert int(fields[3]) == len(want)
    assert float(fields[5]) == float(want[3]["val"][0]) == 0.25  # the ARG t slot carries the time (ir.rs:342-348)
    assert int(fields[7]) == int(want[-1]["opcode_uses"])
