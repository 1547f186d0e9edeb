"""Serving on the GPU: requests that arrive while others run are admitted as
slots and the HBM budget allow, their steps share the device with the
resident scenes, and each result is bit-identical to the same scene stepped
alone (same precision)."""
import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu


def _requests():
    rng = np.random.default_rng(5)
    return [
        (scenes.random_cluster(0, n=40), 9),
        (scenes.settling_box(n_side=4, max_iterations=200), 14),
        (scenes.lattice_container(rng, 200, max_iterations=300), 11),
        (scenes.random_cluster(3, n=27, mu=0.4), 6),
        (scenes.ball_on_ground(h=1e-3), 12),
        (scenes.lattice_container(rng, 120, max_iterations=300), 8),
    ]


def _alone(native, sc, nsteps, precision, **kw):
    g = native.NativeScene.from_scene(sc, precision=precision, **kw)
    g.step(nsteps)
    p, v = g.state()
    g.close()
    return p, v


def _work_alone(native, sc, nsteps, precision, **kw):
    """The solver-work sums a served request reports, from the scene stepped
    alone (per-step history)."""
    g = native.NativeScene.from_scene(sc, precision=precision, **kw)
    g.step(nsteps)
    h = g.history(clear=True)
    g.close()
    w = dict.fromkeys(("iterations", "iteration_contacts", "refine_iterations",
                       "refine_iteration_contacts", "backtracks", "backtrack_contacts",
                       "refined_solves", "refined_contacts"), 0.0)
    for x in h:
        nc = x["num_contacts"]
        if nc == 0:
            continue
        ri, it = x["refine_iterations"], x["iterations"] - x["refine_iterations"]
        w["iterations"] += it
        w["iteration_contacts"] += it * nc
        w["refine_iterations"] += ri
        w["refine_iteration_contacts"] += ri * nc
        w["backtracks"] += x["backtracks"]
        w["backtrack_contacts"] += x["backtracks"] * nc
        if ri > 0:
            w["refined_solves"] += 1
            w["refined_contacts"] += nc
    return w


def _serve(native, reqs, precision, budget=150e9, max_active=4096, steps_per_round=3,
           max_bodies=0, **kw):
    srv = native.NativeServer(precision=precision, hbm_budget_bytes=budget, max_active=max_active,
                              steps_per_round=steps_per_round, max_resident_bodies=max_bodies)
    ids = []
    results = {}
    max_resident = 0
    # staggered arrivals: two at once, then one per round, then the rest together
    arrivals = [[0, 1], [2], [], [3], [4, 5]]
    busy = True
    r = 0
    while busy or r < len(arrivals):
        if r < len(arrivals):
            for i in arrivals[r]:
                if i < len(reqs):
                    ids.append((i, srv.submit(reqs[i][0], reqs[i][1], **kw)))
        busy = srv.round()
        max_resident = max(max_resident, srv.stats()["active"])
        for res in srv.poll():
            results[res["id"]] = res
        r += 1
        assert r < 500
    states = {i: srv.result_state(rid) for i, rid in ids}
    st = srv.stats()
    srv.close()
    return ids, results, states, st, max_resident


@pytest.mark.parametrize("precision,refine", [(0, 0), (1, 0), (1, 500)],
                         ids=["fp64", "mixed", "mixed_refined"])
def test_served_results_equal_alone(native, precision, refine):
    reqs = _requests()
    kw = {"refine_iterations": refine} if refine else {}
    ids, results, states, st, _ = _serve(native, reqs, precision, **kw)
    assert st["completed"] == len(reqs) and st["pending"] == 0 and st["active"] == 0
    for i, rid in ids:
        res = results[rid]
        assert res["status"] == 0
        assert res["nsteps"] == reqs[i][1]
        assert res["t_admit"] >= res["t_submit"] and res["t_done"] >= res["t_admit"]
        assert 0 <= res["solves_at_tolerance"] <= res["solves"] <= res["nsteps"]
        p, v = _alone(native, reqs[i][0], reqs[i][1], precision, **kw)
        ps, vs = states[i]
        assert np.array_equal(ps, p) and np.array_equal(vs, v), i
        w = _work_alone(native, reqs[i][0], reqs[i][1], precision, **kw)
        for key, val in w.items():
            assert res[key] == val, (i, key)
    if refine:
        assert sum(results[rid]["refined_solves"] for _, rid in ids) > 0


def test_served_ragged_requests_equal_alone(native):
    """A single free sphere, only fixed boxes, one sphere overlapped by 40
    others, a ball on the ground and a cluster, served together: each result
    equals the scene stepped alone; the contact-free ones report no solve."""
    grav = scenes.default_params(gravity=(0.0, 0.0, -9.81))
    one = scenes._assemble([], np.array([[0.0, 0.0, 1.0]]), np.array([0.05]), 2600.0,
                           dict(grav), "one_sphere")
    walls = scenes._assemble(scenes.open_box(1.0, 1.0, 1.0), np.zeros((0, 3)), np.zeros(0),
                             2600.0, dict(grav), "walls_only")
    reqs = [(one, 7), (scenes.crowd(40), 5), (walls, 4), (scenes.ball_on_ground(h=1e-3), 9),
            (scenes.random_cluster(0, n=40), 6)]
    ids, results, states, st, _ = _serve(native, reqs, 0)
    assert st["completed"] == len(reqs)
    for i, rid in ids:
        res = results[rid]
        assert res["status"] == 0 and res["nsteps"] == reqs[i][1]
        p, v = _alone(native, reqs[i][0], reqs[i][1], 0)
        ps, vs = states[i]
        assert np.array_equal(ps, p) and np.array_equal(vs, v), i
        if i in (0, 2):
            assert res["solves"] == 0, i


def test_request_over_the_partner_limit_is_retired_alone(native):
    """A request whose scene goes over the pair kernels' partner limit (a
    gridded sphere with 8,193 partners, scenes.raspberry) fails the step for
    every resident scene; the server retires that request with DV_ERR_ARG and
    no steps done, and the others are served to the end, each equal to the
    scene stepped alone."""
    reqs = [(scenes.random_cluster(0, n=40), 6), (scenes.raspberry(8193, ballast=8200), 4),
            (scenes.ball_on_ground(h=1e-3), 9)]
    ids, results, states, st, _ = _serve(native, reqs, 0)
    assert st["completed"] == len(reqs)
    for i, rid in ids:
        res = results[rid]
        if i == 1:
            assert res["status"] == 1 and res["nsteps"] == 0
            continue
        assert res["status"] == 0 and res["nsteps"] == reqs[i][1]
        p, v = _alone(native, reqs[i][0], reqs[i][1], 0)
        ps, vs = states[i]
        assert np.array_equal(ps, p) and np.array_equal(vs, v), i


def test_budget_limits_residency(native):
    reqs = _requests()
    nb_max = max(sc.nb for sc, _ in reqs)
    # room for about two of the larger scenes at a time (about 2.5 kB per body)
    budget = 2.2 * 2.5e3 * nb_max
    ids, results, states, st, max_resident = _serve(native, reqs, 1, budget=budget)
    assert st["completed"] == len(reqs)
    assert max_resident <= 3
    for i, rid in ids:
        p, v = _alone(native, reqs[i][0], reqs[i][1], 1)
        assert np.array_equal(states[i][0], p), i


def test_max_active_one_is_sequential(native):
    reqs = _requests()[:3]
    ids, results, states, st, max_resident = _serve(native, reqs, 0, max_active=1)
    assert max_resident == 1 and st["completed"] == 3
    order = sorted(results.values(), key=lambda r: r["t_admit"])
    for a, b in zip(order, order[1:]):
        assert b["t_admit"] >= a["t_done"]


def test_resident_body_limit(native):
    """max_resident_bodies bounds the bodies stepped together (the work of a
    step): at every admission the requests admitted and not yet finished hold
    at most that many bodies, unless one request alone is larger; results stay
    the same bits as alone."""
    reqs = _requests()
    cap = 150
    ids, results, states, st, _ = _serve(native, reqs, 1, max_bodies=cap)
    assert st["completed"] == len(reqs)
    res = list(results.values())
    for r in res:
        t = r["t_admit"]
        resident = [q for q in res if q["t_admit"] <= t < q["t_done"]]
        if len(resident) > 1:
            assert sum(q["nb"] for q in resident) <= cap, (t, [(q["id"], q["nb"]) for q in resident])
    assert max(r["nb"] for r in res) > cap  # one request is admitted alone
    for i, rid in ids:
        p, v = _alone(native, reqs[i][0], reqs[i][1], 1)
        assert np.array_equal(states[i][0], p), i


def test_segment_count_growing_within_capacity(native):
    """Admissions that raise the resident count without outgrowing the segment
    capacity (100 resident, then 101 -- capacity 125 --, then 121) keep the
    per-step records in bounds: every result is the same bits as alone."""
    balls = [scenes.free_balls(n=1 + (i % 3), tolerance=1e-6) for i in range(121)]
    srv = native.NativeServer(precision=0, max_active=4096, steps_per_round=2)
    ids = []
    for stage in (range(0, 100), range(100, 101), range(101, 121)):
        for i in stage:
            ids.append((i, srv.submit(balls[i], 6)))
        srv.round()
    busy = True
    while busy:
        busy = srv.round()
    srv.poll()
    for i, rid in ids:
        p, v = _alone(native, balls[i], 6, 0)
        ps, vs = srv.result_state(rid)
        assert np.array_equal(ps, p) and np.array_equal(vs, v), i
    srv.close()
