"""PGS on the GPU (System(6), src/PGS.cu:367-459) against the oracle: the
sweep runs in contact order on one thread per scene and the residual is
elementwise or a maximum, so the GPU result is bit-identical."""
import numpy as np
import pytest

from dvide_b200 import scenes, workloads

pytestmark = pytest.mark.gpu


def _pgs(sc, **kw):
    sc.params["solver"] = 6
    sc.params.update(kw)
    return sc


@pytest.mark.parametrize("make", [lambda: scenes.random_cluster(0, n=40),
                                  lambda: scenes.random_cluster(3, n=60, mu=0.45),
                                  lambda: scenes.random_cluster(5, n=27, mu=0.0)])
def test_pgs_teacher_forced_bitexact(native, oracle_mod, make):
    sc = _pgs(make(), max_iterations=3000)
    g = native.NativeScene.from_scene(sc)
    o = oracle_mod.OracleScene(sc)
    solved = 0
    for k in range(8):
        p, v = o.state()
        g.set_state(p, v)
        o.step(1)
        g.step(1)
        so, sg = o.stats(), g.stats()
        assert sg["num_contacts"] == so["num_contacts"], k
        assert np.array_equal(g.state()[1], o.state()[1]), k
        assert np.array_equal(g.state()[0], o.state()[0]), k
        if so["num_contacts"]:
            solved += 1
            assert np.array_equal(g.gamma(), o.gamma()), k
            assert sg["iterations"] == so["iterations"], k
            assert sg["residual"] == so["residual"], k
    assert solved > 0


def test_pgs_free_running_identical(native, oracle_mod):
    sc = _pgs(scenes.settling_box(n_side=5), max_iterations=2000)
    g = native.NativeScene.from_scene(sc)
    o = oracle_mod.OracleScene(sc)
    for _ in range(60):
        o.step(1)
        g.step(1)
    assert np.array_equal(g.state()[0], o.state()[0])
    assert np.array_equal(g.state()[1], o.state()[1])


def test_pgs_sweep_longer_than_one_pass(native, oracle_mod):
    """~39k contacts: each sweep takes two passes of the sequential thread."""
    d = np.load(workloads.COLUMN_FILE)
    order = np.argsort(d["pos"][:, 2])[:11000]
    sc = _pgs(workloads._column_scene(d["pos"][order], d["radius"][order],
                                      float(d["wall_height"])), max_iterations=3)
    g = native.NativeScene.from_scene(sc)
    o = oracle_mod.OracleScene(sc)
    g.step(1)
    o.step(1)
    assert o.stats()["num_contacts"] > 32768
    assert g.stats()["iterations"] == o.stats()["iterations"] == 3
    assert np.array_equal(g.gamma(), o.gamma())
    assert np.array_equal(g.state()[1], o.state()[1])


def test_pgs_batch_equals_alone(native):
    rng = np.random.default_rng(4)
    scs = [_pgs(scenes.random_cluster(1, n=30)), _pgs(scenes.lattice_container(rng, 120)),
           _pgs(scenes.ball_on_ground(h=1e-3)), _pgs(scenes.random_cluster(7, n=50))]
    b = native.NativeBatch(scs)
    b.step(12)
    for i, sc in enumerate(scs):
        g = native.NativeScene.from_scene(sc)
        g.step(12)
        assert np.array_equal(b.state(i)[0], g.state()[0]), i
        assert np.array_equal(b.gamma(i), g.gamma()), i
        g.close()


def test_pgs_mixed_precision_is_refused(native):
    sc = _pgs(scenes.random_cluster(1, n=30))
    with pytest.raises(Exception):
        native.NativeScene.from_scene(sc, precision=native.DV_PREC_MIXED)
