"""The C++ layer's headers (include/dvide/*.h) compile the programs written
against them -- the settle driver and the test programs that the GPU tests
run -- with warnings as errors, on the CPU; and the uploads of System::p_d,
v_d and gamma_d accept the containers the reference's drivers use."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
PROGRAMS = [os.path.join(ROOT, "dvide_b200", "drivers", "settle.cpp"),
            os.path.join(ROOT, "tests", "cxx", "io_roundtrip.cpp"),
            os.path.join(ROOT, "tests", "cxx", "shear_moves.cpp")]

ASSIGNMENTS = r"""
#include <array>
#include <deque>
#include <vector>
#include "dvide/System.h"
// the assignments drivers write (the System is never initialised here: only
// that they compile is checked)
void moves(System* sys, const std::vector<double>& p0, const std::deque<double>& v,
           const std::array<double, 6>& g) {
  std::vector<double> f = sys->f_contact_d;  // download
  sys->p_d = p0;                             // upload from a std::vector
  sys->v_d = v;                              // ... or any container of doubles
  sys->gamma_d = g;
  sys->v_d = sys->v_d;                       // values, not the handle
  (void)f;
}
"""


def _syntax(src, extra=()):
    return subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-Werror",
                           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
                           *extra, src], capture_output=True, text=True)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
@pytest.mark.parametrize("src", PROGRAMS, ids=lambda p: os.path.basename(p))
def test_programs_compile_against_the_headers(src):
    out = _syntax(src)
    assert out.returncode == 0, out.stderr[-3000:]


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_device_array_assignments_compile(tmp_path):
    src = tmp_path / "moves.cpp"
    src.write_text(ASSIGNMENTS)
    out = _syntax(str(src))
    assert out.returncode == 0, out.stderr[-3000:]
