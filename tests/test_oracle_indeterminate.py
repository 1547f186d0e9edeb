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


def _warm_cold_spread(oracle_mod, sc, steps):
    """Largest relative gamma difference, per step, between the FP64 oracle's
    own (warm-started) solve and a cold-started FP64 solve of the same step."""
    o = oracle_mod.OracleScene(sc)
    worst = 0.0
    for _ in range(steps):
        p, v = o.state()
        g = o.gamma()
        cold = oracle_mod.OracleScene(sc)
        cold.set_state(p, v)
        cold.set_gamma(np.zeros_like(g))
        o.step(1)
        cold.step(1)
        go = o.gamma()
        if o.stats()["num_contacts"] and np.abs(go).max() > 0:
            worst = max(worst, float(np.linalg.norm(cold.gamma() - go) / np.linalg.norm(go)))
    return worst


def test_scenes_whose_fp64_gamma_is_pinned(oracle_mod):
    """The scenes the mixed-precision gamma bound (1e-5 relative) is held on:
    at tolerance 1e-8 a warm- and a cold-started FP64 solve of every step agree
    to well within that bound (a sliding ball, a 5-sphere stack in motion,
    the 40-sphere cluster), while a 10-sphere stack does not (the smallest
    eigenvalue of N of a chain falls like 1 / n^2)."""
    ball = scenes.ball_on_ground(h=1e-2, tolerance=1e-8, warm_start=1)
    ball.vel[1] = (0.2, 0.0, 0.1)
    assert _warm_cold_spread(oracle_mod, ball, 5) < 1e-6
    stack = scenes.sphere_stack(5, tolerance=1e-8)
    stack.vel[1:] = (0.1, 0.0, -0.05)
    assert _warm_cold_spread(oracle_mod, stack, 20) < 1e-5
    cluster = scenes.random_cluster(0, n=40, max_iterations=20000, tolerance=1e-8)
    assert _warm_cold_spread(oracle_mod, cluster, 8) < 1e-6
    chain = scenes.sphere_stack(10, tolerance=1e-8)
    chain.vel[1:] = (0.1, 0.0, -0.05)
    assert _warm_cold_spread(oracle_mod, chain, 20) > 1e-5
