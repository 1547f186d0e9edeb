"""PGJ on the GPU (System(5), src/PGJ.cu:152-224) against the oracle: every
quantity is elementwise or a maximum, so the GPU result is bit-identical."""
import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu


def _pgj(sc, **kw):
    sc.params["solver"] = 5
    sc.params.update(kw)
    return sc


@pytest.mark.parametrize("make", [lambda: scenes.random_cluster(0, n=40),
                                  lambda: scenes.random_cluster(3, n=60, mu=0.45)])
def test_pgj_teacher_forced_bitexact(native, oracle_mod, make):
    sc = _pgj(make(), max_iterations=3000)
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
        pg, vg = g.state()
        po, vo = o.state()
        assert np.array_equal(vg, vo) and np.array_equal(pg, po), k
        if so["num_contacts"]:
            solved += 1
            assert np.array_equal(g.gamma(), o.gamma()), k
            assert sg["iterations"] == so["iterations"], k
            assert sg["residual"] == so["residual"], k
    assert solved > 0


def test_pgj_free_running_identical(native, oracle_mod):
    sc = _pgj(scenes.settling_box(n_side=5), max_iterations=2000)
    g = native.NativeScene.from_scene(sc)
    o = oracle_mod.OracleScene(sc)
    for _ in range(60):
        o.step(1)
        g.step(1)
    assert np.array_equal(g.state()[0], o.state()[0])
    assert np.array_equal(g.state()[1], o.state()[1])


def test_pgj_batch_equals_alone(native):
    rng = np.random.default_rng(4)
    scs = [_pgj(scenes.random_cluster(1, n=30)), _pgj(scenes.lattice_container(rng, 120)),
           _pgj(scenes.ball_on_ground(h=1e-3))]
    b = native.NativeBatch(scs)
    b.step(12)
    for i, sc in enumerate(scs):
        g = native.NativeScene.from_scene(sc)
        g.step(12)
        assert np.array_equal(b.state(i)[0], g.state()[0]), i


def test_mixed_solver_batch_rejected(native):
    a = scenes.random_cluster(1, n=20)
    b = _pgj(scenes.random_cluster(2, n=20))
    with pytest.raises(native.DvError):
        native.NativeBatch([a, b])
