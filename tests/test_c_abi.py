"""The C ABI from a C program: include/boxzy_gpu.h and boxzy_diag.h compile as
C99 with warnings as errors, the program links against libboxzy_gpu.so, and the
entry points that need no device answer as documented (version string, ghost-fill
plan, adjoint checkpoint plan, parameter refusals with bx_last_error)."""
import os
import shutil
import subprocess

import pytest

from boxzyhydro_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r"""
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "boxzy_gpu.h"
#include "boxzy_diag.h"

int main(void) {
  printf("version %s\n", bx_version());
  bx_params p;
  memset(&p, 0, sizeof p);
  p.nx = 12; p.ny = 10; p.nz = 8; p.h2stat = -1;
  p.dx = p.dy = p.dz = 0.1; p.cfl = 0.4; p.gammafix = 1.4;
  p.small_rho = 1e-12; p.small_eps = 1e-40; p.vlimit = 10.0;
  int64_t nghost = 0;
  int32_t fused_ok = -1;
  if (bx_ghost_plan(&p, &nghost, NULL, NULL, NULL, NULL, NULL, &fused_ok) != BX_OK) return 2;
  int32_t *dst = malloc(nghost * sizeof *dst), *src = malloc(nghost * sizeof *src);
  uint8_t *sgn = malloc(nghost);
  if (bx_ghost_plan(&p, &nghost, dst, src, sgn, NULL, NULL, NULL) != BX_OK) return 3;
  printf("ghosts %lld fused %d first %d last %d\n", (long long)nghost, (int)fused_ok,
         (int)dst[0], (int)dst[nghost - 1]);
  int64_t first = -1, again = -1;
  int32_t chain = -1;
  if (bx_adj_plan(200, 15, &first, &again, &chain) != BX_OK) return 4;
  printf("plan %lld %lld %d\n", (long long)first, (long long)again, (int)chain);
  bx_handle *h = NULL;
  p.nx = 4;
  int rc = bx_create(&p, &h);
  printf("create %d %s %s\n", rc, h ? "handle" : "null", bx_last_error(NULL));
  free(dst); free(src); free(sgn);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_program_against_the_header_and_library(tmp_path):
    src = tmp_path / "abi.c"
    src.write_text(SRC)
    exe = tmp_path / "abi"
    libdir = os.path.dirname(_lib.LIB_PATH)
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
           "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
           "-L", libdir, "-lboxzy_gpu", f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = dict(line.split(" ", 1) for line in out.stdout.strip().splitlines())
    assert "sm_100a" in lines["version"]
    ng = 12 * 10 * 8 - 8 * 6 * 4  # cells minus the interior
    assert lines["ghosts"].split()[:3] == [str(ng), "fused", "1"]
    assert lines["plan"] == "232 429 15"
    assert lines["create"].startswith("1 null grid too small")
