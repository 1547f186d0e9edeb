"""Warm starts in the CPU oracle: positional (the reference's resize
semantics, parity mode) and matched by contact pair (warm_start 2, opt-in)."""
import numpy as np

from dvide_b200 import scenes


def test_matched_equals_positional_on_an_unchanging_list(oracle_mod):
    res = []
    for ws in (1, 2):
        sc = scenes.ball_on_ground(warm_start=ws)
        o = oracle_mod.OracleScene(sc)
        o.step(4)
        res.append((o.stats()["iterations"], o.gamma(), o.state()[1]))
    assert res[0][0] == res[1][0]
    assert np.array_equal(res[0][1], res[1][1]) and np.array_equal(res[0][2], res[1][2])


def test_matched_start_is_the_pairs_previous_impulse(oracle_mod):
    """After the list shifts (a low-id sphere leaves), a matched step equals a
    positional step whose warm start was mapped pair by pair by hand."""
    sc = scenes.random_cluster(0, n=64, tolerance=1e-7, max_iterations=5000)
    sc.params["warm_start"] = 2
    a = oracle_mod.OracleScene(sc)
    a.step(3)
    old_a, old_b, _, _ = a.contacts()
    old_g = a.gamma()
    p, v = a.state()
    p[5] += np.array([0.0, 0.0, 50.0])  # the first sphere after the five boxes
    v[5] = 0.0
    a.set_state(p, v)
    # the reference: a positional solve started from the hand-mapped impulses
    sc_b = scenes.random_cluster(0, n=64, tolerance=1e-7, max_iterations=5000)
    sc_b.params["warm_start"] = 1
    b = oracle_mod.OracleScene(sc_b)
    b.set_state(p, v)
    b.collide()
    new_a, new_b, _, _ = b.contacts()
    old = {(int(x), int(y)): g for x, y, g in zip(old_a, old_b, old_g)}
    g0 = np.array([old.get((int(x), int(y)), np.zeros(3)) for x, y in zip(new_a, new_b)])
    assert 0 < sum((int(x), int(y)) in old for x, y in zip(new_a, new_b)) < len(new_a)
    b.set_gamma(g0)
    a.step(1)
    b.step(1)
    assert a.stats()["iterations"] == b.stats()["iterations"]
    assert np.array_equal(a.gamma(), b.gamma())
    assert np.array_equal(a.state()[1], b.state()[1])
