"""include/dvide.h is a C header: a C99 program compiles against it with
-pedantic -Werror, links libdvide_b200.so and runs the calls that need no GPU
(defaults, status strings, argument checks)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "dvide.h"

int main(void) {
  dv_params p;
  dv_scene* s = NULL;
  if (dv_params_default(&p) != DV_OK) return 1;
  if (p.h != 1e-3 || p.mu != 0.25 || p.solver != DV_SOLVER_APGD || p.fp64_narrowphase != 0)
    return 2;
  /* no bodies: rejected before any device use */
  if (dv_scene_create(NULL, 0, &p, &s) == DV_OK) return 3;
  if (dv_params_default(NULL) != DV_ERR_ARG) return 4;
  printf("%s\n", dv_status_string(DV_ERR_ARG));
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_compiles_as_c99_and_links(native, tmp_path):
    src = tmp_path / "use_dvide.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "use_dvide"
    libdir = os.path.join(ROOT, "dvide_b200")
    cmd = ["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
           "-L", libdir, "-ldvide_b200", f"-Wl,-rpath,{libdir}"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, (run.returncode, run.stderr)
    assert run.stdout.strip()
