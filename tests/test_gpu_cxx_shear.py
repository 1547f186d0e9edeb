"""Bodies moved between steps the way the reference's shear and draft drivers
move them (models/test_shear.cu:378-406, models/test_draft.cu:438-439), through
the C++ layer (include/dvide/System.h): System::p_d and v_d written from host
vectors after DoTimeStep.  tests/cxx/shear_moves.cpp runs the driver's loop
(a fixed wall pushed in at 0.2 m/s, one sphere held in x and z, positions
re-integrated from the step's start); the oracle replays the same sequence
from the bodies the program wrote, and every step's contact and iteration
counts and the final positions and velocities must be identical.  The
program also checks the uploads' errors."""
import os
import subprocess

import numpy as np
import pytest

from dvide_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dvide_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")

pytestmark = pytest.mark.gpu

STEPS = 150
WALL, HELD = 2, 35  # the +x wall; a sphere of the top layer


@pytest.fixture(scope="module")
def run(tmp_path_factory):
    d = tmp_path_factory.mktemp("shear")
    exe = str(d / "shear_moves")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(CUDA, "include"),
                           os.path.join(HERE, "cxx", "shear_moves.cpp"), "-o", exe, "-L", PKG,
                           "-ldvide_cxx", "-ldvide_b200", "-L", os.path.join(CUDA, "lib64"),
                           "-lcudart", f"-Wl,-rpath,{PKG}"])
    out = subprocess.run([exe, str(d), str(STEPS)], capture_output=True, text=True, timeout=300)
    return d, out


def test_upload_errors(run):
    d, out = run
    assert out.returncode == 0, out.stdout + out.stderr
    assert "upload checks: early 1 sized 1 output 1" in out.stdout
    assert "gamma kept: 1" in out.stdout


def test_driver_moves_replayed_by_the_oracle(run, oracle_mod):
    d, out = run
    assert out.returncode == 0, out.stdout + out.stderr
    rows = [l for l in out.stdout.splitlines() if l and l[0].isdigit()]
    driver = [(int(l.split(",")[1]), int(l.split(",")[2])) for l in rows]
    assert len(driver) == STEPS
    b = np.loadtxt(d / "shear_initial.txt")
    h = 1e-3
    params = scenes.default_params(h=h, gravity=(0.0, 0.0, -9.81), tolerance=1e-6,
                                   max_iterations=500, warm_start=1)
    sc = scenes.Scene(b[:, 0:3].copy(), b[:, 3:6].copy(), b[:, 6].copy(), b[:, 7:10].copy(),
                      b[:, 10].astype(np.int32), np.full(len(b), -1, dtype=np.int32), params,
                      "shear_moves")
    assert sc.fixed[WALL] == 1 and sc.fixed[HELD] == 0
    o = oracle_mod.OracleScene(sc)
    replay = []
    on_wall = 0
    for s in range(STEPS):
        p0, _ = o.state()
        assert o.step(1) == 0, s
        st = o.stats()
        replay.append((st["num_contacts"], st["iterations"]))
        a, bb = o.contacts()[:2]
        on_wall = max(on_wall, int(np.count_nonzero((a == WALL) | (bb == WALL))))
        _, v = o.state()
        v[WALL] = (-0.2, 0.0, 0.0)
        v[HELD, 0] = 0.0
        v[HELD, 2] = 0.0
        o.set_state(h * v + p0, v)
        if s == STEPS // 2:
            o.set_gamma(o.gamma())
    assert driver == replay
    assert on_wall > 0 and max(c for c, _ in replay) > 30
    final = np.loadtxt(d / "shear_final.txt")
    p, v = o.state()
    assert np.array_equal(final[:, 0:3], p) and np.array_equal(final[:, 3:6], v)
