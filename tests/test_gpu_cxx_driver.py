"""The C++ layer (include/dvide/System.h) runs a driver written like the
reference's models/test_compaction.cu and gives the oracle's trajectory: the
driver writes the bodies it built at full precision, the oracle replays the
same scene, and every step's contact count and iteration count and the final
positions and velocities must be identical."""
import os
import subprocess

import numpy as np
import pytest

from dvide_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "dvide_b200", "drivers", "settle")

pytestmark = pytest.mark.gpu


def _replay(oracle_mod, tmp_path, steps, tolerance, max_iterations, warm_start, solver=1,
            rows=(), anti_relaxation=0):
    """The driver's scene (settle_initial.txt) with the driver's settings
    (System defaults: mu 0.25, envelope 1e-3; h 1e-3, gravity -z) in the oracle."""
    b = np.loadtxt(tmp_path / "settle_initial.txt")
    params = scenes.default_params(h=1e-3, gravity=(0.0, 0.0, -9.81), tolerance=tolerance,
                                   max_iterations=max_iterations, warm_start=warm_start,
                                   solver=solver, anti_relaxation=anti_relaxation)
    sc = scenes.Scene(b[:, 0:3].copy(), b[:, 3:6].copy(), b[:, 6].copy(), b[:, 7:10].copy(),
                      b[:, 10].astype(np.int32), np.full(len(b), -1, dtype=np.int32), params,
                      "settle_driver")
    o = oracle_mod.OracleScene(sc)
    for row in rows:
        o.add_bilateral(*row)
    per_step = []
    for _ in range(steps):
        o.step(1)
        st = o.stats()
        per_step.append((st["num_contacts"], st["iterations"]))
    return o, per_step


def test_settle_driver_runs(tmp_path, oracle_mod):
    out = subprocess.run([DRIVER, "120", "1", "1e-4", "1000"], cwd=tmp_path, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l and l[0].isdigit()]
    assert len(lines) == 120
    last = [float(x) for x in lines[-1].split(",")]
    assert last[1] > 100          # contacts once the lattice has landed
    assert os.path.exists(tmp_path / "settle_final.csv")
    rows = open(tmp_path / "settle_final.csv").read().splitlines()
    assert rows[0].startswith("1005,") and len(rows) == 1006
    assert "contact handles: ok" in out.stdout
    # the oracle's trajectory, step by step and at the end, bit for bit
    o, per_step = _replay(oracle_mod, tmp_path, 120, 1e-4, 1000, 1)
    driver = [(int(l.split(",")[1]), int(l.split(",")[2])) for l in lines]
    assert driver == per_step
    final = np.loadtxt(tmp_path / "settle_final_full.txt")
    p, v = o.state()
    assert np.array_equal(final[:, 0:3], p) and np.array_equal(final[:, 3:6], v)


def test_unsupported_solver_type_reports(tmp_path):
    out = subprocess.run([DRIVER, "1", "2", "1e-4"], cwd=tmp_path, capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 1
    assert "unsupported" in out.stderr


@pytest.mark.parametrize("args", [["5", "1e-3", "2000"], ["6", "1e-4", "3000"],
                                  ["1", "1e-4", "1000", "2"]],
                         ids=["pgj", "pgs", "apgd_matched_warm_start"])
def test_settle_driver_other_solver_forms(tmp_path, oracle_mod, args):
    """System(5) (PGJ), System(6) (PGS) and APGD with the warm start matched by
    contact pair, through the C++ layer: the oracle's trajectory, bit for bit.
    The System passes warm_start 0 to PGJ and PGS, which start from (1, 0, 0)."""
    out = subprocess.run([DRIVER, "120", *args], cwd=tmp_path, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l and l[0].isdigit()]
    assert len(lines) == 120
    last = [float(x) for x in lines[-1].split(",")]
    assert last[1] > 100
    assert all(np.isfinite(float(x)) for x in lines[-1].split(","))
    solver = int(args[0])
    warm = int(args[3]) if len(args) > 3 else (1 if solver == 1 else 0)
    o, per_step = _replay(oracle_mod, tmp_path, 120, float(args[1]), int(args[2]), warm,
                          solver=solver)
    driver = [(int(l.split(",")[1]), int(l.split(",")[2])) for l in lines]
    assert driver == per_step
    final = np.loadtxt(tmp_path / "settle_final_full.txt")
    p, v = o.state()
    assert np.array_equal(final[:, 0:3], p) and np.array_equal(final[:, 3:6], v)



def test_settle_driver_with_pinned_spheres(tmp_path, oracle_mod):
    """System::addBilateralConstraintDOF through the C++ layer: the x and y
    DOFs of a column of 10 spheres stay where they started while the pile
    settles around them, and the run is the oracle's with the same rows."""
    out = subprocess.run([DRIVER, "120", "1", "1e-4", "1000", "1", "10"], cwd=tmp_path,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l and l[0].isdigit()]
    assert len(lines) == 120
    drift = [l for l in out.stdout.splitlines() if l.startswith("pinned drift:")]
    assert len(drift) == 1
    assert float(drift[0].split(":")[1]) < 1e-5
    # the oracle with the same rows (x, then y, of spheres 5..14), bit for bit
    rows = [(3 * (5 + i) + k, -1) for i in range(10) for k in range(2)]
    o, per_step = _replay(oracle_mod, tmp_path, 120, 1e-4, 1000, 1, rows=rows)
    driver = [(int(l.split(",")[1]), int(l.split(",")[2])) for l in lines]
    assert driver == per_step
    final = np.loadtxt(tmp_path / "settle_final_full.txt")
    p, v = o.state()
    assert np.array_equal(final[:, 0:3], p) and np.array_equal(final[:, 3:6], v)


def test_settle_driver_anti_relaxation(tmp_path, oracle_mod):
    """APGD::setAntiRelaxation through the C++ layer: the oracle's trajectory
    with anti-relaxation, bit for bit."""
    out = subprocess.run([DRIVER, "80", "1", "1e-4", "1000", "1", "0", "1"], cwd=tmp_path,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l and l[0].isdigit()]
    assert len(lines) == 80
    o, per_step = _replay(oracle_mod, tmp_path, 80, 1e-4, 1000, 1, anti_relaxation=1)
    driver = [(int(l.split(",")[1]), int(l.split(",")[2])) for l in lines]
    assert driver == per_step
    assert max(c for c, _ in per_step) > 100
    final = np.loadtxt(tmp_path / "settle_final_full.txt")
    p, v = o.state()
    assert np.array_equal(final[:, 0:3], p) and np.array_equal(final[:, 3:6], v)


def _mm(path):
    with open(path) as f:
        head = f.readline()
        dims = [int(x) for x in f.readline().split()]
        body = [l.split() for l in f if l.strip()]
    return head, dims, body


def test_export_matrices(tmp_path):
    """System::exportMatrices (System.cu:1912-1934), as models/test_compaction.cu
    calls it: D (3 nc + nbil rows, 3 nb columns, 18 entries per contact and 1
    per single-DOF row), Minv, r, b, k of the last step."""
    out = subprocess.run([DRIVER, "30", "1", "1e-4", "1000", "1", "3"], cwd=tmp_path,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    nc = int([l for l in out.stdout.splitlines() if l and l[0].isdigit()][-1].split(",")[1])
    nbil, nb = 6, 1005
    head, dims, body = _mm(tmp_path / "D.mtx")
    assert head.startswith("%%MatrixMarket matrix coordinate real general")
    assert dims == [3 * nc + nbil, 3 * nb, 18 * nc + nbil] and len(body) == dims[2]
    rows = np.array([int(b[0]) for b in body])
    assert np.all(np.diff(rows) >= 0) and rows.min() == 1 and rows.max() == 3 * nc + nbil
    head, dims, body = _mm(tmp_path / "Minv.mtx")
    assert dims == [3 * nb, 3 * nb, 3 * nb]
    assert all(float(b[2]) == 0.0 for b in body[:15])  # the five fixed boxes
    for name, n in (("r", 3 * nc + nbil), ("b", 3 * nc + nbil), ("k", 3 * nb)):
        head, dims, body = _mm(tmp_path / f"{name}.mtx")
        assert head.startswith("%%MatrixMarket matrix array real general")
        assert dims == [n, 1] and len(body) == n
        assert all(np.isfinite(float(b[0])) for b in body)
