"""Bilateral DOF rows (System::addBilateralConstraintDOF, System.cu:510-532,
622-638, 1526-1544) in the CPU oracle: known answers from the constraint's
definition, and the reference's own conventions (no projection, the residual
without contacts, the flat initial guess)."""
import numpy as np
import pytest

from dvide_b200 import scenes

G = 9.81


def test_pinned_dof_holds_its_position(oracle_mod):
    """A free sphere whose z DOF is pinned (DOFB < 0) keeps z at its initial
    value while x stays in free flight; the row's impulse carries the weight:
    gamma = m g h (a bilateral row is never projected)."""
    sc = scenes.free_balls(1, vel=[[0.3, 0.0, 0.0]])
    sc.bilateral = [(2, -1, 0.0, 0.0)]
    o = oracle_mod.OracleScene(sc)
    z0 = sc.pos[0, 2]
    for _ in range(20):
        o.step(1)
        assert o.stats()["num_contacts"] == 0
        p, v = o.state()
        assert abs(p[0, 2] - z0) < 1e-9 and abs(v[0, 2]) < 1e-8
    assert np.isclose(p[0, 0], sc.pos[0, 0] + 20 * 1e-3 * 0.3, rtol=0, atol=1e-12)
    g = o.bilateral_gamma()
    assert g.shape == (1,)
    assert np.isclose(g[0], sc.mass[0] * G * 1e-3, rtol=1e-6)
    assert np.allclose(o.fcontact()[0], [0.0, 0.0, sc.mass[0] * G], rtol=1e-6)


def test_prescribed_velocity(oracle_mod):
    """b = (p - p0 - velocity (t - t_start)) / h, velocity 0 before t_start:
    the step that starts at time t leaves the DOF at p0 + velocity (t - t_start)."""
    h, vel, ts = 1e-3, 0.5, 0.01
    sc = scenes.free_balls(1, h=h)
    sc.bilateral = [(0, -1, vel, ts)]
    o = oracle_mod.OracleScene(sc)
    x0 = sc.pos[0, 0]
    t = 0.0
    for _ in range(40):
        o.step(1)
        p, _ = o.state()
        target = x0 + (vel * (t - ts) if t >= ts else 0.0)
        assert abs(p[0, 0] - target) < 1e-9
        t += h


def test_coupled_pair(oracle_mod):
    """x_1 - x_2 (DOFA, DOFB; no p0: System.cu:1537-1539 drives p_A - p_B to
    0): two equal spheres at equal x moving apart in x stop (momentum zero
    conserved); y and z unaffected."""
    sc = scenes.free_balls(2, vel=[[0.2, 0.1, 0.0], [-0.2, 0.0, 0.0]])
    sc.pos[1] = [0.0, 0.5, 1.0]
    sc.bilateral = [(0, 3, 0.0, 0.0)]
    o = oracle_mod.OracleScene(sc)
    for _ in range(5):
        o.step(1)
        p, v = o.state()
        assert abs(v[0, 0] - v[1, 0]) < 1e-8 and abs(v[0, 0] + v[1, 0]) < 1e-8
        assert abs(p[0, 0] - p[1, 0]) < 1e-9
    assert np.isclose(v[0, 1], 0.1) and np.isclose(v[1, 1], 0.0)


def test_coupled_pair_closes_its_gap(oracle_mod):
    """A two-DOF row at distance d: one step moves the DOFs together
    (v_A - v_B = -d / h), momentum conserved."""
    sc = scenes.free_balls(2)
    sc.pos[1] = [0.01, 0.5, 1.0]
    sc.bilateral = [(0, 3, 0.0, 0.0)]
    o = oracle_mod.OracleScene(sc)
    o.step(1)
    p, v = o.state()
    assert abs(p[0, 0] - p[1, 0]) < 1e-9
    assert np.isclose(v[0, 0] - v[1, 0], 0.01 / 1e-3, rtol=1e-9)
    assert abs(v[0, 0] + v[1, 0]) < 1e-8


def test_rows_with_contacts_keep_equilibrium(oracle_mod):
    """A cluster with pinned, coupled and moving DOFs: the solve converges, the
    pinned DOF stays put, the coupled DOFs coincide."""
    sc = scenes.bilateral_cluster(0, tolerance=1e-7, max_iterations=20000)
    o = oracle_mod.OracleScene(sc)
    (pin, _, _, _), (ca, cb, _, _) = sc.bilateral[0], sc.bilateral[1]
    z0 = sc.pos[pin // 3, pin % 3]
    for _ in range(5):
        assert o.step(1) == 0
        st = o.stats()
        assert st["num_contacts"] > 0 and st["residual"] < 1e-7
    p, _ = o.state()
    assert abs(p[pin // 3, pin % 3] - z0) < 1e-7
    assert abs(p[ca // 3, ca % 3] - p[cb // 3, cb % 3]) < 1e-7
    assert o.bilateral_gamma().shape == (4,)


def test_rows_only_residual_is_the_plain_gradient(oracle_mod):
    """Without contacts getResidual skips the projection and both axpby
    (APGD.cu:96-100): the solve of a single pinned DOF stops once |N x + r|
    is below the tolerance, the same count for any positive gdiff."""
    sc = scenes.free_balls(1, tolerance=1e-4)
    sc.bilateral = [(2, -1, 0.0, 0.0)]
    o = oracle_mod.OracleScene(sc)
    o.step(1)
    st = o.stats()
    assert st["status"] == 0 and st["residual"] < 1e-4
    # N = 1/m, r = -g h: |N x + r| of the returned x
    g = o.bilateral_gamma()[0]
    assert abs(g / sc.mass[0] - G * 1e-3) <= st["residual"] + 1e-15


def test_flat_initial_guess_without_warm_start(oracle_mod):
    """With the warm start off the first iterate is not zero: the reference's
    initialiser writes (1, 0, 0) over flat entries [0, 3 nc) of a vector whose
    first entries are the bilateral rows (APGD.cu:114-120, 200).  After one
    iteration the two starts differ; converged, they agree."""
    res = {}
    for ws in (0, 1):
        for iters in (1, 20000):
            sc = scenes.ball_on_ground(warm_start=ws, tolerance=1e-10)
            sc.params["max_iterations"] = iters
            # 5 consistent rows on the ball's x and z (body 1, at x = z = 0;
            # gravity and the contact act in y): nbil = 5 > 3 nc = 3
            sc.bilateral = [(3, -1, 0.0, 0.0), (5, -1, 0.0, 0.0), (3, 5, 0.0, 0.0),
                            (5, 3, 0.0, 0.0), (3, -1, 0.0, 0.0)]
            o = oracle_mod.OracleScene(sc)
            o.step(1)
            assert o.stats()["num_contacts"] == 1
            res[ws, iters] = o.state()[1]
    assert not np.array_equal(res[0, 1], res[1, 1])
    assert np.allclose(res[0, 20000], res[1, 20000], rtol=0, atol=1e-8)


def test_pgj_and_pgs_reject_rows(oracle_mod):
    for solver in (5, 6):
        sc = scenes.free_balls(1)
        sc.params["solver"] = solver
        sc.bilateral = [(2, -1, 0.0, 0.0)]
        o = oracle_mod.OracleScene(sc)
        assert o.step(1) == 4


def test_dof_out_of_range(oracle_mod):
    sc = scenes.free_balls(1)
    o = oracle_mod.OracleScene(sc)
    with pytest.raises(ValueError):
        o.add_bilateral(3)
    with pytest.raises(ValueError):
        o.add_bilateral(-1)


def test_reduce_orders_agree(oracle_mod):
    """The tiled reduction order (rows' tiles after the contacts' tiles) and
    the flat sequential order give the same velocities to solver tolerance (a
    packed frictional cluster is statically indeterminate: the impulses of two
    solves may differ, the velocities do not)."""
    sc = scenes.bilateral_cluster(1, tolerance=1e-10, max_iterations=20000)
    res = []
    for mode in (0, 1):
        o = oracle_mod.OracleScene(sc, reduce_mode=mode)
        o.step(3)
        res.append(o.state()[1])
    assert np.allclose(res[0], res[1], rtol=0, atol=1e-7)
