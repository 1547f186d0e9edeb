"""The System file formats through the C++ layer (include/dvide/System.h):
exportSystem -> importSystem -> steps (System.cu:1699-1737, :1856-1910), the
columns of the System and CollisionDetector files against the reference's
writers (System.cu:1699-1737, CollisionDetector.cu:667-711), the per-contact
force file (System.cu:1259-1295, :1672-1697) and the importer's sphere mass.

tests/cxx/io_roundtrip.cpp does the C++ side; it checks itself that the
imported System equals the exported one bit for bit (bodies, masses, state)
and that both step identically, and writes each file beside a
full-precision dump of the values the file holds."""
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dvide_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")

pytestmark = pytest.mark.gpu

STEPS = 40


def _g(x):
    """A double as the reference's writers print it (stream defaults: %g, six digits)."""
    return "%g" % x


@pytest.fixture(scope="module")
def run(tmp_path_factory):
    d = tmp_path_factory.mktemp("io")
    exe = str(d / "io_roundtrip")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                           "-I", os.path.join(CUDA, "include"),
                           os.path.join(HERE, "cxx", "io_roundtrip.cpp"), "-o", exe, "-L", PKG,
                           "-ldvide_cxx", "-ldvide_b200", "-L", os.path.join(CUDA, "lib64"),
                           "-lcudart", f"-Wl,-rpath,{PKG}"])
    out = subprocess.run([exe, str(d), str(STEPS)], capture_output=True, text=True, timeout=300)
    return d, out


def _rows(path):
    with open(path) as f:
        return [l.rstrip("\n") for l in f]


def test_export_import_step_identical(run):
    d, out = run
    assert out.returncode == 0, out.stdout + out.stderr
    line = [l for l in out.stdout.splitlines() if l.startswith("roundtrip identical")]
    assert line, out.stdout
    assert int(line[0].split()[-2]) > STEPS  # contacts were solved on the way


def test_imported_sphere_mass_is_the_references(run):
    """Every imported sphere gets 2600 * 4 * 3.14159 * pow(r, 3) / 3
    (System.cu:1902), boxes mass 1 -- bit for bit (math.pow is C's pow)."""
    d, out = run
    assert out.returncode == 0
    full = np.loadtxt(d / "a_end_full.txt")
    for (r, m), row in zip(np.loadtxt(d / "masses.txt"), full):
        if row[8] == 0:  # a sphere: geometry (r, 0, 0)
            assert m == 2600 * 4.0 * 3.14159 * math.pow(r, 3.0) / 3.0
        else:
            assert m == 1.0


def test_system_export_columns(run):
    """System::exportSystem rows: index, fixed, p, the unit quaternion 1 0 0 0,
    v, shape code (0 sphere + radius, 2 box + half-extents), each followed by
    ', ', numbers at the stream's default six digits; header: body count and
    three zero counts (beams, plates, 2-D bodies)."""
    d, out = run
    assert out.returncode == 0
    rows = _rows(d / "a_end.csv")
    full = np.loadtxt(d / "a_end_full.txt")
    assert rows[0] == f"{len(full)}, 0, 0, 0, "
    assert len(rows) == len(full) + 1
    for i, (row, x) in enumerate(zip(rows[1:], full)):
        fixed, p, v, g = int(x[0]), x[1:4], x[4:7], x[7:10]
        want = [str(i), str(fixed), *map(_g, p), "1", "0", "0", "0", *map(_g, v)]
        want += ["0", _g(g[0])] if g[1] == 0 else ["2", *map(_g, g)]
        assert row == ", ".join(want) + ", ", (i, row)


def test_collision_detector_export_columns(run):
    """CollisionDetector::exportSystem rows: index, body A, body B, the stored
    normal (B -> A) and gap, then position, velocity and geometry of A and of B."""
    d, out = run
    assert out.returncode == 0
    rows = _rows(d / "cd_end.csv")
    cd = np.loadtxt(d / "cd_end_full.txt", ndmin=2)
    full = np.loadtxt(d / "a_end_full.txt")
    assert len(rows) == len(cd) > 0
    for i, (row, c) in enumerate(zip(rows, cd)):
        a, b = int(c[0]), int(c[1])
        assert a < b
        want = [str(i), str(a), str(b), *map(_g, c[2:6])]
        for body in (a, b):
            want += [*map(_g, full[body, 1:4]), *map(_g, full[body, 4:7]), *map(_g, full[body, 7:10])]
        assert row == ", ".join(want) + ", ", (i, row)


def test_contact_force_file(run):
    """outputContactForcePerCollision(file): header (contacts, bodies, 0, 0, 0),
    then index, A, B, location, normal force, friction force per contact;
    the forces are those calculateContactForcePerCollision leaves."""
    d, out = run
    assert out.returncode == 0
    rows = _rows(d / "forces.csv")
    fr = np.loadtxt(d / "forces_full.txt", ndmin=2)
    cd = np.loadtxt(d / "cd_end_full.txt", ndmin=2)
    full = np.loadtxt(d / "a_end_full.txt")
    assert rows[0] == f"{len(fr)}, {len(full)}, 0, 0, 0, "
    assert len(rows) == len(fr) + 1 == len(cd) + 1
    for i, (row, f, c) in enumerate(zip(rows[1:], fr, cd)):
        fields = row.split(", ")
        assert fields[:3] == [str(i), str(int(c[0])), str(int(c[1]))]
        assert fields[6:12] == [_g(x) for x in f], (i, row)
        # the normal force lies along the stored normal, the friction across it
        n = c[2:5]
        assert abs(np.dot(f[3:6], n)) <= 1e-6 * (np.linalg.norm(f[3:6]) + 1e-300)
        assert np.linalg.norm(np.cross(f[0:3], n)) <= 1e-6 * (np.linalg.norm(f[0:3]) + 1e-300)
