"""APGD anti-relaxation (APGD::setAntiRelaxation; APGD.cu:335-345, 104-112)
in the CPU oracle: the fused sequence shared with the GPU and the literal
reference sequence give the same solves, and the option changes them."""
import numpy as np

from dvide_b200 import scenes


def _run(oracle_mod, ar, mode, steps=4):
    sc = scenes.random_cluster(2, n=60, tolerance=1e-7, max_iterations=20000)
    sc.params["anti_relaxation"] = ar
    o = oracle_mod.OracleScene(sc, apgd_mode=mode)
    st = []
    for _ in range(steps):
        assert o.step(1) == 0
        st.append(o.stats())
    return o.state()[1], st


def test_fused_equals_literal_sequence(oracle_mod):
    vf, sf = _run(oracle_mod, 1, 0)
    vl, sl = _run(oracle_mod, 1, 1)
    for a, b in zip(sf, sl):
        assert a["iterations"] == b["iterations"] and a["backtracks"] == b["backtracks"]
        assert np.isclose(a["objective"], b["objective"], rtol=1e-9)
        assert np.isclose(a["residual"], b["residual"], rtol=1e-6)
    assert np.allclose(vf, vl, rtol=0, atol=1e-12)


def test_option_changes_the_solve(oracle_mod):
    v0, s0 = _run(oracle_mod, 0, 0, steps=2)
    v1, s1 = _run(oracle_mod, 1, 0, steps=2)
    assert not np.array_equal(v0, v1)
    assert s0[-1]["objective"] != s1[-1]["objective"]
