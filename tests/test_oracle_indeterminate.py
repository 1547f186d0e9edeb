"""A settled pile is statically indeterminate: two FP64 solves of the same
step that both reach the tolerance, started from different impulses, agree on
the velocities but not on gamma.  This bounds what a gamma comparison between
two solvers (the mixed-precision path against FP64, for one) can show."""
import numpy as np

from dvide_b200 import scenes


def test_two_fp64_solves_differ_in_gamma_not_in_velocity(oracle_mod):
    sc = scenes.settling_box(tolerance=1e-6)
    o = oracle_mod.OracleScene(sc)
    o.step(400)
    p, v = o.state()
    g = o.gamma()
    res = {}
    for warm in (1, 0):
        s2 = scenes.settling_box(tolerance=1e-6, warm_start=warm, max_iterations=20000)
        q = oracle_mod.OracleScene(s2)
        q.set_state(p, v)
        if warm:
            q.set_gamma(g)
        q.step(1)
        assert q.stats()["residual"] < 1e-6
        res[warm] = (q.gamma(), q.state()[1])
    (g1, v1), (g0, v0) = res[1], res[0]
    assert np.linalg.norm(g1 - g0) > 1e-5 * np.linalg.norm(g1)
    assert np.abs(v1 - v0).max() < 2e-5
