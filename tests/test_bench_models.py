"""The byte models behind bench.py's roofline fields (CPU only): the served
line's per-request sum (request_bytes_mixed, from the server's solver-work
sums) equals the batched line's per-step model (solve_bytes_mixed) summed
over the same steps, and the mixed model with no FP32 work left is the FP64
model's iteration term; the served line's recorded 60-s run matches its
profile summary."""
import importlib.util
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_request_sum_equals_per_step_model():
    b = _bench()
    rng = np.random.default_rng(3)
    for _ in range(50):
        nb = int(rng.integers(1, 50000))
        steps = int(rng.integers(1, 40))
        per_step = 0
        acc = dict.fromkeys(("iterations", "iteration_contacts", "refine_iterations",
                             "refine_iteration_contacts", "backtracks", "backtrack_contacts",
                             "refined_solves", "refined_contacts"), 0)
        contacts = solves = 0
        for _ in range(steps):
            nc = int(rng.integers(0, 4 * nb)) if rng.random() > 0.2 else 0
            it = int(rng.integers(0, 500))
            ri = int(rng.integers(0, it + 1)) if rng.random() > 0.5 else 0
            bt = int(rng.integers(0, 80))
            per_step += b.solve_bytes_mixed(nc, nb, it, ri, bt)
            if nc == 0:
                continue
            # the server's sums (dv_server.cu): FP32 iterations apart from FP64 ones
            contacts += nc
            solves += 1
            acc["iterations"] += it - ri
            acc["iteration_contacts"] += (it - ri) * nc
            acc["refine_iterations"] += ri
            acc["refine_iteration_contacts"] += ri * nc
            acc["backtracks"] += bt
            acc["backtrack_contacts"] += bt * nc
            if ri > 0:
                acc["refined_solves"] += 1
                acc["refined_contacts"] += nc
        r = dict(acc, nb=nb, nsteps=steps, contact_steps=contacts, solves=solves)
        assert b.request_bytes_mixed(r) == per_step


def test_mixed_model_limits():
    b = _bench()
    nc, nb = 741238, 200005
    # a scene without contacts only updates
    assert b.solve_bytes_mixed(0, nb, 0, 0, 0) == 96 * nb
    # all iterations in FP64: the iteration term is the FP64 model's
    fp64 = b.solve_bytes_mixed(nc, nb, 500, 500, 0) - b.solve_bytes_mixed(nc, nb, 0, 0, 0)
    setup64 = 2 * (136 * nc + 60 * nb)
    assert fp64 == 500 * (440 * nc + 120 * nb) + setup64
    # an FP32 iteration moves less than an FP64 one
    assert b.solve_bytes_mixed(nc, nb, 2, 0, 0) < b.solve_bytes_mixed(nc, nb, 2, 2, 0)


def test_served_specification_record_matches_its_profile():
    """bench.py's SERVED_SPEC_RECORD repeats the recorded 60-s run; its
    figures are the ones profiles/served_poisson_200ps_60s.md gives."""
    b = _bench()
    r = b.SERVED_SPEC_RECORD
    text = open(os.path.join(ROOT, "profiles", "served_poisson_200ps_60s.md")).read()
    assert f"{r['value'] / 1e6:.2f} M" in text
    assert f"{r['device_contact_steps_per_s'] / 1e6:.2f} M" in text
    assert f"({r['speedup_vs_plain']}x)" in text
    assert f"{r['time_per_step_ms']['p50']} / {r['time_per_step_ms']['p99']} ms" in text
    assert f"{r['completion_latency_s']['p50']} / {r['completion_latency_s']['p99']} s" in text
    assert f"{r['peak_resident_gb']} GB" in text
    assert r["source"].split(": ")[1].startswith("profiles/served_poisson_200ps_60s.md")
