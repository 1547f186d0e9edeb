"""Bilateral DOF rows on the GPU (System::addBilateralConstraintDOF,
System.cu:510-532, 622-638, 1526-1544) against the CPU oracle through the C
ABI: bit-exact, step by step, free running (both sides evaluate the same
floating-point sequence, so their trajectories stay identical): contacts,
contact and row impulses, velocities, positions, contact forces, iteration
counts, residuals, objectives and the CCP violation."""
import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu


def _run(native, oracle_mod, sc, steps, min_solved=None):
    g = native.NativeScene.from_scene(sc)
    o = oracle_mod.OracleScene(sc)
    solved = 0
    for k in range(steps):
        assert o.step(1) == 0, k
        g.step(1)
        so, sg = o.stats(), g.stats()
        assert sg["num_contacts"] == so["num_contacts"], k
        ga, gb, _, _ = g.contacts()
        oa, ob, _, _ = o.contacts()
        assert np.array_equal(ga, oa) and np.array_equal(gb, ob), k
        assert np.array_equal(g.bilateral_gamma(), o.bilateral_gamma()), k
        assert np.array_equal(g.gamma(), o.gamma()), k
        pg, vg = g.state()
        po, vo = o.state()
        assert np.array_equal(vg, vo), k
        assert np.array_equal(pg, po), k
        assert np.array_equal(g.fcontact(), o.fcontact()), k
        assert sg["iterations"] == so["iterations"], k
        assert sg["residual"] == so["residual"], k
        assert sg["objective"] == so["objective"], k
        assert sg["backtracks"] == so["backtracks"], k
        assert np.array_equal(g.ccp_violation(), o.ccp_violation()), k
        for x, y in zip(g.step_vectors(), o.step_vectors()):  # r, b (rows first), k
            assert np.array_equal(x, y), k
        solved += 1
    if min_solved is not None:
        assert solved >= min_solved
    return g, o


@pytest.mark.parametrize("seed,warm", [(0, 1), (1, 0), (2, 2)],
                         ids=["positional", "no_warm_start", "matched"])
def test_cluster_with_rows_bitexact(native, oracle_mod, seed, warm):
    """Contacts and rows together: a pinned DOF, a coupled pair, a DOF moved
    at a prescribed velocity from t = 2 h, a row on a fixed body."""
    sc = scenes.bilateral_cluster(seed, n=64, warm_start=warm)
    g, o = _run(native, oracle_mod, sc, 6)
    assert o.stats()["num_contacts"] > 20
    assert g.bilateral_gamma().shape == (4,)


def test_rows_without_contacts_bitexact(native, oracle_mod):
    """nc = 0: the solve runs for the rows alone (System.cu:560) and the
    residual is |N x + r| (APGD.cu:96-100)."""
    sc = scenes.free_balls(3, vel=[[0.3, 0.0, 0.0], [0.0, 0.2, 0.0], [-0.2, 0.0, 0.1]])
    sc.pos[2] = [0.0, 0.5, 1.0]
    sc.bilateral = [(2, -1, 0.0, 0.0), (0, 6, 0.0, 0.0), (4, -1, 0.5, 0.002)]
    g, o = _run(native, oracle_mod, sc, 5)
    assert o.stats()["num_contacts"] == 0
    p, _ = g.state()
    assert abs(p[0, 2] - 1.0) < 1e-9


def test_more_rows_than_contact_entries_no_warm_start(native, oracle_mod):
    """nbil > 3 nc with the warm start off: the flat (1, 0, 0) initial guess
    covers some rows and no contact (APGD.cu:114-120, 200)."""
    sc = scenes.ball_on_ground(warm_start=0, tolerance=1e-9)
    sc.params["max_iterations"] = 3000
    sc.bilateral = [(3, -1, 0.0, 0.0), (5, -1, 0.0, 0.0), (3, 5, 0.0, 0.0),
                    (5, 3, 0.0, 0.0), (3, -1, 0.0, 0.0)]
    _run(native, oracle_mod, sc, 4)


def test_rows_api_rules(native):
    """Rows are added before the first step, to FP64 APGD scenes only; DOFs
    in range."""
    sc = scenes.free_balls(2)
    g = native.NativeScene.from_scene(sc)
    with pytest.raises(native.DvError):
        g.add_bilateral(6)          # DOF past the last body
    g.add_bilateral(2)
    with pytest.raises(native.DvError):
        g.set_params(solver=native.DV_SOLVER_PGJ)
    g.step(1)
    with pytest.raises(native.DvError):
        g.add_bilateral(5)          # after the first step
    m = native.NativeScene.from_scene(sc, precision=native.DV_PREC_MIXED)
    with pytest.raises(native.DvError):
        m.add_bilateral(2)
