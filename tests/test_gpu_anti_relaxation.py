"""APGD anti-relaxation on the GPU (the kAR solve kernel) against the oracle:
bit-exact, free running: impulses, velocities, positions, iterations,
backtracks, residuals and objectives (objectiveCCP with the last r,
APGD.cu:353-354).  And the cases it is not offered for."""
import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,warm", [(2, 1), (7, 0)])
def test_anti_relaxation_bitexact(native, oracle_mod, seed, warm):
    sc = scenes.random_cluster(seed, n=60, warm_start=warm, tolerance=1e-7,
                               max_iterations=3000)
    sc.params["anti_relaxation"] = 1
    g = native.NativeScene.from_scene(sc)
    o = oracle_mod.OracleScene(sc)
    for k in range(6):
        assert o.step(1) == 0
        g.step(1)
        so, sg = o.stats(), g.stats()
        assert sg["num_contacts"] == so["num_contacts"] > 0, k
        assert sg["iterations"] == so["iterations"], k
        assert sg["backtracks"] == so["backtracks"], k
        assert sg["residual"] == so["residual"], k
        assert sg["objective"] == so["objective"], k
        assert np.array_equal(g.gamma(), o.gamma()), k
        pg, vg = g.state()
        po, vo = o.state()
        assert np.array_equal(vg, vo), k
        assert np.array_equal(pg, po), k


def test_anti_relaxation_toggles(native, oracle_mod):
    """Switched on after some steps and off again through dv_set_params."""
    sc = scenes.random_cluster(3, n=40, warm_start=1, tolerance=1e-7, max_iterations=3000)
    g = native.NativeScene.from_scene(sc)
    o = oracle_mod.OracleScene(sc)
    for k, ar in enumerate([0, 1, 1, 0, 1]):
        g.set_params(anti_relaxation=ar)
        o.params = oracle_mod.make_params({**sc.params, "anti_relaxation": ar})
        oracle_mod.lib().or_set_params(o.h, o.params)
        assert o.step(1) == 0
        g.step(1)
        assert g.stats()["objective"] == o.stats()["objective"], k
        assert np.array_equal(g.state()[1], o.state()[1]), k


def test_anti_relaxation_rules(native):
    """FP64 APGD scenes of their own only: not mixed, not PGJ/PGS, not with
    bilateral rows, not in batches, not through dv_apgd_solve."""
    sc = scenes.random_cluster(0, n=30)
    with pytest.raises(native.DvError):
        native.NativeScene.from_scene(sc, precision=native.DV_PREC_MIXED, anti_relaxation=1)
    with pytest.raises(native.DvError):
        native.NativeScene.from_scene(sc, solver=native.DV_SOLVER_PGJ, anti_relaxation=1)
    g = native.NativeScene.from_scene(sc)
    g.add_bilateral(3 * 5)
    with pytest.raises(native.DvError):
        g.set_params(anti_relaxation=1)
    h = native.NativeScene.from_scene(sc, anti_relaxation=1)
    with pytest.raises(native.DvError):
        h.add_bilateral(3 * 5)
    h.collide()
    with pytest.raises(native.DvError):
        h.solve()
    with pytest.raises(native.DvError):
        native.NativeBatch([sc, sc], anti_relaxation=1)
