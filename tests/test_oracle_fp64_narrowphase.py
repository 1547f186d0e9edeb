"""The opt-in FP64 narrowphase (fp64_narrowphase = 1) in the CPU oracle:
normals and sphere gaps at FP64 accuracy instead of the reference's float
square roots, and a solution that differs from parity mode only at that
level."""
import numpy as np

from dvide_b200 import scenes


def _contacts(oracle_mod, sc, steps=2):
    o = oracle_mod.OracleScene(sc)
    o.step(steps)
    o.collide()
    a, b, nP, loc = o.contacts()
    return o, a, b, nP


def _sphere_gaps(sc, o, a, b, nP):
    p, _ = o.state()
    r = sc.geom[:, 0]
    sph = (sc.geom[a, 1] == 0) & (sc.geom[b, 1] == 0)
    d = np.linalg.norm(p[b[sph]] - p[a[sph]], axis=1)
    return nP[sph, 3], d - (r[a[sph]] + r[b[sph]])


def test_fp64_normals_and_gaps(oracle_mod):
    sc = scenes.random_cluster(4, n=60)
    sc.params["fp64_narrowphase"] = 1
    o, a, b, nP = _contacts(oracle_mod, sc)
    assert len(a) > 20
    norm = np.linalg.norm(nP[:, :3], axis=1)
    assert np.max(np.abs(norm - 1.0)) < 4e-16
    gap, ref = _sphere_gaps(sc, o, a, b, nP)
    assert np.max(np.abs(gap - ref)) < 1e-16 * 10


def test_parity_mode_carries_float_error(oracle_mod):
    sc = scenes.random_cluster(4, n=60)
    o, a, b, nP = _contacts(oracle_mod, sc)
    norm = np.linalg.norm(nP[:, :3], axis=1)
    assert np.max(np.abs(norm - 1.0)) > 1e-10   # float normalisation
    gap, ref = _sphere_gaps(sc, o, a, b, nP)
    assert np.max(np.abs(gap - ref)) > 1e-12


def test_modes_agree_to_float_accuracy(oracle_mod):
    res = []
    for mode in (0, 1):
        sc = scenes.random_cluster(6, n=50, tolerance=1e-8, max_iterations=3000)
        sc.params["fp64_narrowphase"] = mode
        o = oracle_mod.OracleScene(sc)
        o.step(1)
        res.append((o.contacts()[0], o.gamma(), o.state()[1]))
    assert np.array_equal(res[0][0], res[1][0])          # same contact set
    g0, g1 = res[0][1], res[1][1]
    assert not np.array_equal(g0, g1)
    assert np.linalg.norm(g0 - g1) <= 1e-4 * np.linalg.norm(g0)
    v0, v1 = res[0][2], res[1][2]
    assert np.linalg.norm(v0 - v1) <= 1e-4 * np.linalg.norm(v0)
