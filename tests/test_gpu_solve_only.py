"""The solver's own solve() (dv_apgd_solve; APGD::solve, PGJ::solve,
PGS::solve through the C++ layer): the step's solve on the current state and
the last collision detection's contacts, without the update, bit-identical
to the oracle's `or_solve`; a step after it continues from its warm start
exactly as the oracle does."""
import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu


def _scene(kind):
    if kind == "apgd":
        return scenes.random_cluster(4, n=60, warm_start=1)
    if kind == "apgd_rows":
        return scenes.bilateral_cluster(5, n=64, warm_start=1)
    sc = scenes.random_cluster(6, n=40, warm_start=0)
    sc.params["solver"] = 5 if kind == "pgj" else 6
    sc.params["max_iterations"] = 2000
    return sc


@pytest.mark.parametrize("kind", ["apgd", "apgd_rows", "pgj", "pgs"])
def test_solve_alone_bitexact(native, oracle_mod, kind):
    sc = _scene(kind)
    g = native.NativeScene.from_scene(sc)
    o = oracle_mod.OracleScene(sc)
    o.step(2)
    g.step(2)
    o.collide()
    g.collide()
    p0, v0 = o.state()
    t0 = g.stats()["time"]
    assert o.solve() == 0
    assert g.solve() == 0
    so, sg = o.stats(), g.stats()
    assert sg["num_contacts"] == so["num_contacts"] > 0
    assert sg["iterations"] == so["iterations"]
    assert sg["residual"] == so["residual"]
    assert sg["objective"] == so["objective"]
    assert np.array_equal(g.gamma(), o.gamma())
    assert np.array_equal(g.bilateral_gamma(), o.bilateral_gamma())
    pg, vg = g.state()
    po, vo = o.state()
    assert np.array_equal(pg, p0) and np.array_equal(po, p0)  # no update
    assert np.array_equal(vg, vo)
    if kind != "pgs":  # PGS works on System::v, as the reference's
        assert np.array_equal(vg, v0)
    assert g.stats()["time"] == t0
    # the next step starts from this solve's warm start on both sides
    o.step(1)
    g.step(1)
    assert np.array_equal(g.gamma(), o.gamma())
    assert np.array_equal(g.state()[1], o.state()[1])
    assert np.array_equal(g.state()[0], o.state()[0])
