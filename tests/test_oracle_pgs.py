"""PGS (System(6), src/PGS.cu) in the CPU oracle: known answers."""
import numpy as np

from dvide_b200 import scenes


def test_pgs_ball_carries_its_weight(oracle_mod):
    """models/test_oneBall.cu: a unit ball resting on a fixed box; the normal
    impulse per step converges to m g h = 9.81e-2."""
    sc = scenes.ball_on_ground()
    sc.params["solver"] = 6
    o = oracle_mod.OracleScene(sc)
    for _ in range(3):
        o.step(1)
        st = o.stats()
        assert st["num_contacts"] == 1 and st["residual"] < 1e-4
        g = o.gamma()
        assert abs(g[0, 0] - 9.81e-2) < 5e-4 and abs(g[0, 1]) < 1e-12 and abs(g[0, 2]) < 1e-12


def test_pgs_and_apgd_solve_the_same_ccp(oracle_mod):
    """Both solvers minimise the same cone-constrained quadratic: at tight
    tolerances their impulses agree."""
    sc = scenes.random_cluster(0, n=40, tolerance=1e-9, max_iterations=20000)
    res = {}
    for solver in (1, 6):
        sc.params["solver"] = solver
        o = oracle_mod.OracleScene(sc)
        o.step(1)
        res[solver] = (o.gamma(), o.stats())
    g1, g6 = res[1][0], res[6][0]
    assert res[6][1]["residual"] < 1e-9
    assert np.linalg.norm(g1 - g6) <= 1e-6 * np.linalg.norm(g6)


def test_pgs_needs_fewer_sweeps_than_pgj(oracle_mod):
    """Gauss-Seidel uses each update at once; Jacobi waits a sweep."""
    it = {}
    for solver in (5, 6):
        sc = scenes.random_cluster(3, n=60, tolerance=1e-6, max_iterations=50000)
        sc.params["solver"] = solver
        o = oracle_mod.OracleScene(sc)
        o.step(1)
        it[solver] = o.stats()["iterations"]
    assert 0 < it[6] < it[5]


def test_pgs_zero_iterations_keeps_initial_guess(oracle_mod):
    sc = scenes.random_cluster(2, n=27, max_iterations=0)
    sc.params["solver"] = 6
    o = oracle_mod.OracleScene(sc)
    o.step(1)
    g = o.gamma()
    assert o.stats()["iterations"] == 0
    assert np.array_equal(g[:, 0], np.ones(len(g))) and not g[:, 1:].any()
