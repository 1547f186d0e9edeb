#!/usr/bin/env python
"""Contact-steps/s of the DVIDE rigid-body contact step on B200.

Workload (default): the 200,000-sphere column at rest (about 7.41e5 contacts
per step; r ~ U[0.004, 0.006] m, rho 2500, mu 0.3, h 5e-4, APGD tolerance 1e-4,
at most 500 iterations, warm start, plain FP64), loaded from
dvide_b200/data/column_settled.npz.  A step is one System::DoTimeStep:
collision detection, APGD solve, velocity/position update.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm: W untimed steps, then K steps timed with CUDA events on the stream
the library launches on (barrier + synchronize on both sides, max over ranks);
value = contacts summed over the K steps and all ranks / time.  e2e repeats
the same K steps (same starting state and warm start) through the host-buffer
API, the state copied in from pinned memory and back out every step.  Under torchrun every rank runs its own replica of the
scene (no collective on the data path).
Reference arm (--impl reference): the CPU restatement of the reference's
algorithm (oracle/, OpenMP over all host cores) on the same state and
configuration; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


# Compulsory FP64 bytes (structure of arrays, each array touched once):
#   one Schur product N x ........ 136 nc + 60 nb
#   one APGD iteration ........... 440 nc + 120 nb  (two products + vector streams)
#   per extra backtrack .......... one product
#   per step outside the loop .... setup (k, r, the Lipschitz estimate: 2 products),
#                                  final D^T gamma and update: 136 nc + 96 nb
def solve_bytes(nc, nb, sweeps, backtracks):
    bN = 136 * nc + 60 * nb
    return sweeps * (440 * nc + 120 * nb) + backtracks * bN + 2 * bN + (136 * nc + 96 * nb)


# Mixed precision with FP64 refinement (the batched and served forms): FP32
# iterations at the FP32 variant's compulsory bytes, 248 nc + 72 nb each, and
# one FP32 product, 76 nc + 36 nb, per backtrack and for each of the two setup
# products; the FP64 refinement iterations at 440 nc + 120 nb, with the
# refinement launch's own FP64 setup (two products) when a solve is refined;
# then the FP64 update.  A scene without contacts only updates (96 nb).
def solve_bytes_mixed(nc, nb, iterations, refine_iterations, backtracks):
    if nc == 0:
        return 96 * nb
    bN32 = 76 * nc + 36 * nb
    bN64 = 136 * nc + 60 * nb
    it32 = iterations - refine_iterations
    return (it32 * (248 * nc + 72 * nb) + refine_iterations * (440 * nc + 120 * nb)
            + backtracks * bN32 + 2 * bN32 + (2 * bN64 if refine_iterations > 0 else 0)
            + (136 * nc + 96 * nb))


# solve_bytes_mixed summed over a served request's steps, from the sums the
# server reports (dv_request_result).
def request_bytes_mixed(r):
    nb, c = r["nb"], r["contact_steps"]
    return (248 * r["iteration_contacts"] + 72 * nb * r["iterations"]
            + 440 * r["refine_iteration_contacts"] + 120 * nb * r["refine_iterations"]
            + 76 * r["backtrack_contacts"] + 36 * nb * r["backtracks"]
            + 2 * (76 * c + 36 * nb * r["solves"])
            + 2 * (136 * r["refined_contacts"] + 60 * nb * r["refined_solves"])
            + 136 * c + 96 * nb * r["nsteps"])


# The same count for the kernel's own sequence: ONE Schur product per APGD
# iteration (N y is formed from the stored products of the last two iterates),
# i.e. 440 nc + 120 nb less one product's 136 nc + 60 nb.
def solve_bytes_one_product(nc, nb, sweeps, backtracks):
    bN = 136 * nc + 60 * nb
    return sweeps * (304 * nc + 60 * nb) + backtracks * bN + 2 * bN + (136 * nc + 96 * nb)


# DRAM bytes per algorithmic byte of the solve kernel, measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum = 4.371 + 1.994 GB) on a
# 30-iteration launch on this workload (11.415 GB algorithmic); the full launch
# is scaled by it.
TRAFFIC_PER_ALGORITHMIC_BYTE = 6.365664 / 11.415179


def collide_bytes(nc, nb, npossible):
    return 24 * nb + 4 * 16 * nb + 8 * npossible + 8 * npossible + 48 * npossible + nc * (8 + 32 + 72)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def load_workload(name):
    from dvide_b200 import scenes, workloads
    if name == "column":
        sc = workloads.column_settled()
        desc = ("column_settled: 200000 spheres r~U[0.004,0.006] rho 2500 mu 0.3 h 5e-4 "
                "tol 1e-4 maxIter 500 warm start, FP64")
    elif name == "settling":
        sc = scenes.settling_box()
        desc = "settling_box: 1000 spheres r 0.05 rho 2600 mu 0.25 h 1e-3 tol 1e-4 maxIter 1000"
    else:
        raise SystemExit(f"unknown workload {name}")
    return sc, desc


# The reference's APGD as written (src/APGD.cu:164-361): four Schur products
# per iteration, sequential host sums, COO entries in their literal order.
LITERAL = dict(reduce_mode=1, spmv_mode=1, apgd_mode=1)


def run_reference(args, sc, desc):
    """The reference's algorithm on the host cores (oracle/, its literal APGD
    sequence), same state and config; the fused evaluation order the GPU uses,
    timed beside it on one step, as a second number."""
    from oracle import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    o = O.OracleScene(sc, threads=threads, **LITERAL)
    budget = args.ref_budget_s
    contacts = 0
    done = 0
    t0 = time.perf_counter()
    while done < args.steps:
        o.step(1)
        contacts += o.stats()["num_contacts"]
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    dt = time.perf_counter() - t0
    value = contacts / dt
    f = O.OracleScene(sc, threads=threads)
    t1 = time.perf_counter()
    f.step(1)
    dtf = time.perf_counter() - t1
    fused = f.stats()["num_contacts"] / dtf
    at_tol = None
    if args.workload == "column":
        # the compacting column (every step at the tolerance), first steps
        from dvide_b200 import workloads
        c = O.OracleScene(workloads.column_compacting(), threads=threads, **LITERAL)
        ct, cc, cn, its = 0.0, 0, 0, []
        while cn < args.ref_tol_steps:
            t2 = time.perf_counter()
            c.step(1)
            ct += time.perf_counter() - t2
            cc += c.stats()["num_contacts"]
            its.append(c.stats()["iterations"])
            cn += 1
        at_tol = {"value": cc / ct, "unit": "contact-steps/s", "cores": threads,
                  "sample": f"first {cn} of the compacting column's steps ({ct:.1f} s), literal "
                            f"sequence", "iterations": its}
    sample = (f"first {done} of {args.steps} full time steps from the benchmark's initial state "
              f"({dt:.1f} s), {threads} OpenMP threads, the reference's literal APGD sequence "
              f"(four Schur products per iteration, sequential sums)")
    return {"metric": "contact-steps/s", "value": value, "unit": "contact-steps/s",
            "impl": "reference", "n_gpus": 0, "steps": done, "warmup": 0,
            "ms_per_step": 1e3 * dt / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc},
            "cpu_baseline": {"value": value, "unit": "contact-steps/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "column_at_tolerance": at_tol,
            "fused_order_port": {"value": fused, "unit": "contact-steps/s", "cores": threads,
                                 "sample": f"first step, {dtf:.1f} s, one Schur product per "
                                           f"iteration (the GPU's evaluation order)"},
            "e2e": {"value": value, "unit": "contact-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def cpu_baseline_sample(sc, budget_s):
    from oracle import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    o = O.OracleScene(sc, threads=threads, **LITERAL)
    t0 = time.perf_counter()
    contacts = 0
    n = 0
    while True:
        o.step(1)
        contacts += o.stats()["num_contacts"]
        n += 1
        if time.perf_counter() - t0 > budget_s * 0.5 or n >= 50:
            break
    dt = time.perf_counter() - t0
    return {"value": contacts / dt, "unit": "contact-steps/s", "cores": threads, "kind": "port",
            "sample": f"first {n} time step(s) from the same initial state and stored warm "
                      f"start, {dt:.1f} s, the reference's literal APGD sequence"}


def _rel(a, b):
    n = float(np.linalg.norm(b))
    d = float(np.linalg.norm(a - b))
    return d / n if n > 0 else d


def run_mixed_error(N, stream, steps=500, every=10):
    """Mixed precision (FP32 iterates, FP64 sums and update) against FP64 on the
    1,000-sphere settling box (h 1e-3, at most 1000 iterations, warm start):
    every `every`-th of `steps` steps, the mixed solve starts from the FP64
    run's state and warm start and both take one step; relative 2-norm errors
    of gamma and v, the largest velocity difference, and both residuals.  At
    the benchmark tolerance 1e-4 the two solves stop at different iterates, so
    the difference includes the solver tolerance; at 1e-6 it is the precision.
    The settling box is statically indeterminate once it rests (gamma is not
    unique there); `determinate` holds the scenes whose FP64 gamma is pinned.
    The FP64 path gives the oracle's results bit for bit
    (tests/test_gpu_parity.py)."""
    from dvide_b200 import scenes

    out = {"workload": (f"settling_box 1000 spheres, every {every}th of {steps} steps "
                        f"(teacher-forced from the FP64 run), h 1e-3, maxIter 1000")}
    for tol, refine in ((1e-4, 0), (1e-6, 0), (1e-6, 2000)):
        sc = scenes.settling_box(tolerance=tol)
        f = N.NativeScene.from_scene(sc)
        m = N.NativeScene.from_scene(sc, precision=N.DV_PREC_MIXED, refine_iterations=refine)
        f.set_stream(stream.cuda_stream)
        m.set_stream(stream.cuda_stream)
        rows = []
        for k in range(steps):
            if (k + 1) % every:
                f.step(1)
                continue
            p, v = f.state()
            m.set_state(p, v)
            m.set_gamma(f.gamma())
            f.step(1)
            m.step(1)
            sf, sm = f.stats(), m.stats()
            if sf["num_contacts"] == 0:
                continue
            vf, vm = f.state()[1], m.state()[1]
            rows.append((_rel(m.gamma(), f.gamma()), _rel(vm, vf), float(np.abs(vm - vf).max()),
                         sf["residual"], sm["residual"], sf["iterations"], sm["iterations"],
                         sm["refine_iterations"]))
        f.close()
        m.close()
        if not rows:
            continue
        a = np.array(rows)
        key = f"tolerance_{tol:g}" + ("_fp64_refinement" if refine else "")
        out[key] = {
            "steps_compared": len(rows),
            "gamma_rel_err": {"max": float(a[:, 0].max()), "median": float(np.median(a[:, 0]))},
            "v_rel_err": {"max": float(a[:, 1].max()), "median": float(np.median(a[:, 1]))},
            "v_abs_err_max_m_per_s": float(a[:, 2].max()),
            "residual_fp64_max": float(a[:, 3].max()),
            "residual_mixed_max": float(a[:, 4].max()),
            "iterations_mean": {"fp64": float(a[:, 5].mean()), "mixed": float(a[:, 6].mean())},
        }
        if refine:
            out[key]["fp64_refinement_iterations_mean"] = float(a[:, 7].mean())
    out["determinate"] = run_mixed_determinate(N, stream)
    return out


def run_mixed_determinate(N, stream, tol=1e-8, refine=2000):
    """Mixed precision on scenes whose FP64 gamma is pinned at tolerance 1e-8
    (a warm- and a cold-started FP64 solve of the same step agree to < 1e-5;
    tests/test_oracle_indeterminate.py): a ball sliding on the ground, a
    5-sphere stack dropping and sliding, the 40-sphere cluster.  Teacher-forced
    from the FP64 run; the mixed solve with FP64 refinement (up to `refine`
    FP64 iterations from the FP32 best iterate once the FP32 phase stalls) and
    without it.  Cost: device time per step of each."""
    from dvide_b200 import scenes

    def scene(which):
        if which == "ball_sliding":
            sc = scenes.ball_on_ground(h=1e-2, tolerance=tol, warm_start=1)
            sc.vel[1] = (0.2, 0.0, 0.1)
            return sc, 5
        if which == "stack5_moving":
            sc = scenes.sphere_stack(5, tolerance=tol)
            sc.vel[1:] = (0.1, 0.0, -0.05)
            return sc, 20
        return scenes.random_cluster(0, n=40, max_iterations=5000, tolerance=tol), 8

    out = {"tolerance": tol, "bound": "gamma and v within 1e-5 relative of FP64"}
    for which in ("ball_sliding", "stack5_moving", "cluster40"):
        sc, steps = scene(which)
        f = N.NativeScene.from_scene(sc)
        forms = {"mixed": N.NativeScene.from_scene(sc, precision=N.DV_PREC_MIXED),
                 "mixed_refined": N.NativeScene.from_scene(sc, precision=N.DV_PREC_MIXED,
                                                           refine_iterations=refine)}
        for g in [f, *forms.values()]:
            g.set_stream(stream.cuda_stream)
        acc = {k: {"g": 0.0, "v": 0.0, "res": 0.0, "it": [], "rit": [], "ms": []} for k in forms}
        fms = []
        for _ in range(steps):
            p, v = f.state()
            gam = f.gamma()
            for g in forms.values():
                g.set_state(p, v)
                g.set_gamma(gam)
            f.step(1)
            sf = f.stats()
            if sf["num_contacts"] == 0:
                continue
            fms.append(sf["elapsed_ms"])
            gf, vf = f.gamma(), f.state()[1]
            for k, g in forms.items():
                g.step(1)
                sg = g.stats()
                a = acc[k]
                a["g"] = max(a["g"], _rel(g.gamma(), gf))
                a["v"] = max(a["v"], _rel(g.state()[1], vf))
                a["res"] = max(a["res"], sg["residual"])
                a["it"].append(sg["iterations"] - sg["refine_iterations"])
                a["rit"].append(sg["refine_iterations"])
                a["ms"].append(sg["elapsed_ms"])
        row = {"steps": len(fms), "fp64_ms_per_step": float(np.mean(fms)) if fms else None}
        for k, a in acc.items():
            row[k] = {"gamma_rel_err_max": a["g"], "v_rel_err_max": a["v"],
                      "residual_max": a["res"],
                      "fp32_iterations_mean": float(np.mean(a["it"])) if a["it"] else 0.0,
                      "fp64_refinement_iterations_mean": float(np.mean(a["rit"])) if a["rit"] else 0.0,
                      "ms_per_step": float(np.mean(a["ms"])) if a["ms"] else None}
        out[which] = row
        for g in [f, *forms.values()]:
            g.close()
    return out


def run_column_at_tolerance(args, N, torch, stream):
    """The 200,000-sphere column while it compacts (workloads.column_compacting:
    the state from which the next 10 steps all reach the APGD tolerance 1e-4
    within the 500-iteration cap, ~7.29e5 contacts), stepped through those 10
    steps with the benchmark's own settings: contact-steps/s at residual 1e-4,
    with the iterations each step needed.  The kernels are warm (the headline
    ran first)."""
    from dvide_b200 import workloads
    sc = workloads.column_compacting()
    g = N.NativeScene.from_scene(sc)
    g.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.step(args.tol_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    hist = g.history(clear=True)
    g.close()
    contacts = sum(h["num_contacts"] for h in hist)
    tol = sc.params["tolerance"]
    conv = [h for h in hist if h["residual"] < tol]
    conv_ms = sum(h["elapsed_ms"] for h in conv)
    return {
        "converged_steps_only": ({"value": sum(h["num_contacts"] for h in conv) / (conv_ms / 1e3),
                                  "unit": "contact-steps/s", "steps": len(conv)}
                                 if conv and len(conv) < len(hist) else None),
        "workload": (f"column_compacting: the 200000-sphere column while it compacts, "
                     f"{args.tol_steps} steps from the saved state, tol {tol:g} maxIter "
                     f"{sc.params['max_iterations']} warm start, FP64"),
        "value": contacts / (ms / 1e3), "unit": "contact-steps/s", "ms_per_step": ms / len(hist),
        "contacts_per_step": contacts / len(hist),
        "iterations": [h["iterations"] for h in hist],
        "backtracks": [h["backtracks"] for h in hist],
        "residual_max": max(h["residual"] for h in hist),
        "steps_at_tolerance": f"{sum(1 for h in hist if h['residual'] < tol)}/{len(hist)}",
    }


def run_batched(args, N, torch, stream):
    """512 independent settling scenes (sphere counts log-uniform in [100, 20000],
    r ~ U[0.004, 0.006], mu ~ U[0.1, 0.5], own containers; h 1e-3, tol 1e-4,
    maxIter 500, warm start) stepped as one batch: mixed precision, CUDA-graph
    replay, autotuned launch shape.  Beside it, the plain FP64 path stepping a
    size-stratified sample of the same scenes one at a time."""
    from dvide_b200 import scenes
    scs = scenes.batch_scenes(seed=3, count=args.batch_scenes)
    total_steps = args.batch_steps
    timed = max(1, min(args.batch_timed, total_steps - 1))
    pre = total_steps - timed
    b = N.NativeBatch(scs, precision=N.DV_PREC_MIXED, refine_iterations=args.refine)
    b.set_stream(stream.cuda_stream)
    graph = b.set_graph(True) == 0
    b.step(pre)
    tune = b.autotune(steps_per_trial=2)
    torch.cuda.synchronize()
    l0 = b.launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(timed)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    hist, step_ms = b.history()
    contacts = sum(s["num_contacts"] for st in hist for s in st)
    iters = [s["iterations"] for st in hist for s in st if s["num_contacts"] > 0]
    res = [s["residual"] for st in hist for s in st if s["num_contacts"] > 0]
    conv = sum(1 for r in res if r < 1e-4)
    launches = b.launches() - l0
    nb = b.nb
    b.close()
    # roofline over the whole step (collision included; the solve launches are
    # most of it), bytes from every scene's own iteration counts
    nbs = [sc.nb for sc in scs]
    moved = sum(solve_bytes_mixed(x["num_contacts"], nbs[i], x["iterations"],
                                  x["refine_iterations"], x["backtracks"])
                for st in hist for i, x in enumerate(st))
    peak, peak_kind = _peaks()
    achieved = moved / timed / (ms / timed / 1e3) / 1e9
    refine_its = sum(x["refine_iterations"] for st in hist for x in st)
    # plain FP64 path, one scene at a time, on a size-stratified sample
    order = np.argsort([sc.nb for sc in scs])
    sample = [scs[i] for i in order[::max(1, len(scs) // args.plain_sample)]]
    p_contacts = 0
    p_ms = 0.0
    for sc in sample:
        g = N.NativeScene.from_scene(sc)
        g.set_stream(stream.cuda_stream)
        g.step(pre)
        g.history(clear=True)
        g.step(timed)
        h = g.history(clear=True)
        p_contacts += sum(x["num_contacts"] for x in h)
        p_ms += sum(x["elapsed_ms"] for x in h)
        g.close()
    batched = contacts / (ms / 1e3)
    plain = p_contacts / (p_ms / 1e3) if p_ms > 0 else None
    return {
        "workload": (f"{len(scs)} settling scenes, {nb} bodies, steps {pre + 1}-{total_steps} of "
                     f"{total_steps} timed (h 1e-3), mixed precision with up to {args.refine} FP64 "
                     f"refinement iterations, per-scene convergence"),
        "value": batched, "unit": "contact-steps/s", "ms_per_step": ms / timed,
        "contacts_per_step": contacts / timed,
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                       "p99": float(np.percentile(step_ms, 99))},
        "scene_iterations_mean": float(np.mean(iters)) if iters else 0.0,
        "scene_refine_iterations_total": int(refine_its),
        "scene_solves_converged": f"{conv}/{len(res)}",
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                     "kernel": "the whole batched step: FP32 solve launch, FP64 refinement "
                               "launch and collision detection",
                     "bytes_per_step": moved / timed,
                     "bytes_model": "compulsory bytes: FP32 iterations 248 nc + 72 nb, FP64 "
                                    "refinement iterations 440 nc + 120 nb, per scene"},
        "graph": graph, "autotune": {"best": tune["candidates"][tune["best"]],
                                      "identical": tune["identical"]},
        "gpu_launches": int(launches),
        "plain_fp64_one_at_a_time": {
            "value": plain, "unit": "contact-steps/s",
            "sample": f"{len(sample)} of {len(scs)} scenes (every {len(scs) // len(sample)}th by "
                      f"size), same steps, device time"},
        "speedup_vs_plain": (batched / plain) if plain else None,
    }


# The served stream at its specification (Poisson 200/s for 60 s, 12,000
# requests), recorded on one B200 with --serve-seconds 60; the default run
# serves a 1-s window of the same stream and reports this record beside it.
SERVED_SPEC_RECORD = {
    "workload": "12000 requests, Poisson 200/s for 60 s, 200 steps each (h 1e-3), spheres "
                "log-uniform [500, 50000], mixed precision with up to 500 FP64 refinement "
                "iterations, 150 GB budget",
    "value": 21.16e6, "unit": "contact-steps/s (wall clock, arrivals included)",
    "device_contact_steps_per_s": 23.27e6, "speedup_vs_plain": 11.7,
    "time_per_step_ms": {"p50": 1317, "p99": 2260},
    "completion_latency_s": {"p50": 479, "p99": 683},
    "peak_resident_gb": 101.7, "completed": 12000,
    "source": "recorded, not measured in this run: profiles/served_poisson_200ps_60s.md "
              "(python bench.py --steps 3 --warmup 3 --no-batched --no-mixed-error "
              "--no-column-at-tolerance --no-cpu-baseline --serve-seconds 60)",
}


def run_served(args, N, stream):
    """Poisson arrivals of settling scenes (sphere counts log-uniform in
    [500, 50000], r ~ U[0.004, 0.006], mu ~ U[0.1, 0.5], own containers),
    each asking for `serve_steps` steps at h 1e-3 with residual 1e-4, served by
    continuous batching in mixed precision under a 150 GB admission budget.
    Arrivals run in real time.  Beside it, the plain FP64 path serving a
    size-stratified sample of the same requests one at a time."""
    from dvide_b200 import scenes
    rng = np.random.default_rng(11)
    n_req = max(1, int(args.serve_rate * args.serve_seconds))
    gaps = rng.exponential(1.0 / args.serve_rate, size=n_req)
    arrive = np.cumsum(gaps) - gaps[0]
    sizes = np.exp(rng.uniform(np.log(500), np.log(50000), size=n_req)).astype(np.int64)
    # the request scenes are generated in order by a producer thread, a bounded
    # number ahead of their arrival (a long stream does not fit in host memory
    # at once, and generating it in the serving loop would delay the rounds)
    import queue
    import threading
    ahead = queue.Queue(maxsize=min(n_req, 512))

    def produce():
        for j, n in enumerate(sizes):
            ahead.put(scenes.lattice_container(rng, int(n), name=f"req{j}"))

    threading.Thread(target=produce, daemon=True).start()
    while ahead.qsize() < min(n_req, 512):
        time.sleep(0.01)
    srv = N.NativeServer(precision=N.DV_PREC_MIXED, hbm_budget_bytes=150e9,
                         steps_per_round=args.serve_round, keep_states=False,
                         max_resident_bodies=args.serve_max_bodies)
    srv.set_stream(stream.cuda_stream)
    sampler = ClockSampler(torch_device_index())
    sampler.start()
    t0 = time.perf_counter()
    i = 0
    results = []
    busy = False
    trace = []  # (seconds, requests waiting, requests resident, bytes resident) after each round
    next_mark = 0.0
    while i < n_req or busy:
        now = time.perf_counter() - t0
        while i < n_req and arrive[i] <= now:
            srv.submit(ahead.get(), args.serve_steps, refine_iterations=args.refine)
            i += 1
        if not busy and i < n_req and arrive[i] > now:
            time.sleep(min(arrive[i] - now, 0.01))
            busy = srv.stats()["active"] > 0 or srv.stats()["pending"] > 0
            continue
        busy = srv.round()
        results += srv.poll()
        if now >= next_mark:
            st = srv.stats()
            trace.append((round(now, 2), int(st["pending"]), int(st["active"]),
                          float(st["bytes_in_use"])))
            next_mark = now + args.serve_trace_s
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    results += srv.poll()
    st = srv.stats()
    srv.close()
    lat = np.array([r["t_done"] - r["t_submit"] for r in results])
    step_p50 = np.array([r["step_ms_p50"] for r in results])
    step_p99 = np.array([r["step_ms_p99"] for r in results])
    contact_steps = st["contact_steps"]
    # plain FP64 one request at a time on a stratified sample (rebuilt from the
    # same generator: the requests were handed over)
    rng2 = np.random.default_rng(11)
    rng2.exponential(1.0 / args.serve_rate, size=n_req)
    rng2.uniform(np.log(500), np.log(50000), size=n_req)
    order = np.argsort(sizes)
    pick = set(order[::max(1, n_req // args.plain_sample)].tolist())
    sample_reqs = {}
    for j, n in enumerate(sizes):
        sc_j = scenes.lattice_container(rng2, int(n), name=f"req{j}")
        if j in pick:
            sample_reqs[j] = sc_j
    p_cs, p_ms = 0.0, 0.0
    for j in sorted(pick):
        g = N.NativeScene.from_scene(sample_reqs[j])
        g.set_stream(stream.cuda_stream)
        g.step(args.serve_steps)
        h = g.history(clear=True)
        p_cs += sum(x["num_contacts"] for x in h)
        p_ms += sum(x["elapsed_ms"] for x in h)
        g.close()
    plain = p_cs / (p_ms / 1e3) if p_ms > 0 else None
    served = contact_steps / wall
    peak, peak_kind = _peaks()
    moved = sum(request_bytes_mixed(r) for r in results)
    achieved = moved / (st["device_ms"] / 1e3) / 1e9 if st["device_ms"] > 0 else 0.0
    return {
        "workload": (f"{n_req} requests, Poisson {args.serve_rate}/s for {args.serve_seconds} s, "
                     f"{args.serve_steps} steps each (h 1e-3), spheres log-uniform [500, 50000], "
                     f"mixed precision with up to {args.refine} FP64 refinement iterations, "
                     f"150 GB budget"
                     + (f", at most {args.serve_max_bodies} resident bodies"
                        if args.serve_max_bodies else "")),
        "value": served, "unit": "contact-steps/s (wall clock, arrivals included)",
        "device_contact_steps_per_s": contact_steps / (st["device_ms"] / 1e3),
        "wall_s": wall, "completed": int(st["completed"]), "rounds": int(st["rounds"]),
        "layout_changes": int(st["reconfigures"]),
        "time_per_step_ms": {"p50": float(np.percentile(step_p50, 50)),
                             "p99": float(np.percentile(step_p99, 99))},
        "completion_latency_s": {"p50": float(np.percentile(lat, 50)),
                                 "p99": float(np.percentile(lat, 99))},
        "scene_solves_at_tolerance": (f"{sum(r['solves_at_tolerance'] for r in results)}/"
                                      f"{sum(r['solves'] for r in results)}"),
        "backlog": {"max_waiting": max(t[1] for t in trace) if trace else 0,
                    "max_resident": max(t[2] for t in trace) if trace else 0,
                    "peak_resident_gb": max(t[3] for t in trace) / 1e9 if trace else 0.0,
                    "trace_s_waiting_resident_gb": [(t[0], t[1], t[2], round(t[3] / 1e9, 2))
                                                    for t in trace]},
        "plain_fp64_one_at_a_time": {
            "value": plain, "unit": "contact-steps/s (device time)",
            "sample": f"{len(pick)} of {n_req} requests (every {max(1, n_req // args.plain_sample)}th "
                      f"by size)"},
        "speedup_vs_plain": (served / plain) if plain else None,
        "window": ("the whole specification" if args.serve_seconds >= 60 else
                   f"a sample: the first {args.serve_seconds:g} s of arrivals of the 60-s "
                   f"specification (--serve-seconds 60 runs it whole)"),
        "specification_record": None if args.serve_seconds >= 60 else SERVED_SPEC_RECORD,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                     "kernel": "every served step's device time: FP32 solve launch, FP64 "
                               "refinement launch and collision detection",
                     "bytes_model": "compulsory bytes of the batched line, summed per request "
                                    "from the server's per-request solver counts"},
        "clocks": clocks,
    }


def torch_device_index():
    import torch
    return torch.cuda.current_device()


def _oracle_timed_steps(O, threads, sc, states, mode):
    """Steps the oracle once from each (p, v, gamma) in `states` (one step each,
    teacher-forced), timing only the step; returns per-step (contacts,
    seconds, iterations, residual)."""
    o = O.OracleScene(sc, threads=threads, **mode)
    rows = []
    for p, v, gam in states:
        o.set_state(p, v)
        o.set_gamma(gam)
        t = time.perf_counter()
        o.step(1)
        dt = time.perf_counter() - t
        st = o.stats()
        rows.append((st["num_contacts"], dt, st["iterations"], st["residual"]))
    return rows


def _cpu_row(rows, what):
    c = np.array([r[0] for r in rows], dtype=np.float64)
    t = np.array([r[1] for r in rows])
    return {"sample": what, "contact_steps_per_s": float(c.sum() / t.sum()),
            "steps": len(rows), "seconds": float(t.sum()),
            "step_ms": {"mean": float(1e3 * t.mean()), "p50": float(1e3 * np.percentile(t, 50)),
                        "p99": float(1e3 * np.percentile(t, 99))},
            "iterations_mean": float(np.mean([r[2] for r in rows]))}


def run_cpu_table(args):
    """The CPU baseline of every configuration: the reference's literal APGD
    sequence (oracle/, all host cores), with the GPU's evaluation order beside
    it.  C0 runs all 500 steps from its initial state.  C1 and the samples of
    C3 and C4 step the oracle once from states of the plain FP64 GPU
    trajectory (bit-identical to the oracle's own), so that the CPU time goes
    to the timed steps only."""
    from oracle import oracle as O
    from dvide_b200 import _native as N
    from dvide_b200 import scenes, workloads
    O.build()
    threads = os.cpu_count() or 1
    out = {"cores": threads, "modes": {"literal": "the reference's APGD as written (four Schur "
                                                  "products per iteration, sequential sums)",
                                       "fused": "the GPU's evaluation order (one product)"}}
    try:
        out["lscpu"] = subprocess.run(["lscpu"], capture_output=True, text=True).stdout.splitlines()[:20]
    except Exception:
        pass
    modes = {"literal": LITERAL, "fused": {}}
    # C0: every step from the start
    sc = scenes.settling_box()
    row = {}
    for name, m in modes.items():
        o = O.OracleScene(sc, threads=threads, **m)
        rows = []
        for _ in range(500):
            t = time.perf_counter()
            o.step(1)
            dt = time.perf_counter() - t
            st = o.stats()
            rows.append((st["num_contacts"], dt, st["iterations"], st["residual"]))
        row[name] = _cpu_row(rows, "all 500 steps")
        row[name]["ccp_violation_last"] = o.ccp_violation().tolist()
    out["C0"] = row
    # C1: the headline's first step (the column at rest), and the compacting column
    row = {}
    for key, scc in (("settled", workloads.column_settled()),
                     ("compacting", workloads.column_compacting())):
        states = [(scc.pos, scc.vel, scc.gamma)]
        row[key] = {name: _cpu_row(_oracle_timed_steps(O, threads, scc, states, m), "first step")
                    for name, m in modes.items()}
    out["C1"] = row

    def gpu_states(sc, steps, keep):
        g = N.NativeScene.from_scene(sc)
        st = []
        for k in range(steps):
            if k in keep:
                p, v = g.state()
                st.append((p, v, g.gamma()))
            g.step(1)
        g.close()
        return st

    # C3: every 32nd of the 512 scenes by size, steps 61-100 (every 4th)
    scs = scenes.batch_scenes(seed=3, count=512)
    order = np.argsort([x.nb for x in scs])
    rows = {k: [] for k in modes}
    keep = set(range(60, 100, 4))
    for i in order[::32]:
        st = gpu_states(scs[i], 100, keep)
        for name, m in modes.items():
            rows[name] += _oracle_timed_steps(O, threads, scs[i], st, m)
    out["C3"] = {k: _cpu_row(r, "16 of 512 scenes (every 32nd by size), one at a time, "
                                "steps 61-100 (every 4th)") for k, r in rows.items()}
    # C4: 16 requests of the served stream (stratified by size), 200 steps (every 10th)
    rng = np.random.default_rng(11)
    n_req = 12000
    rng.exponential(1.0 / 200.0, size=n_req)
    sizes = np.exp(rng.uniform(np.log(500), np.log(50000), size=n_req)).astype(np.int64)
    pick = set(np.argsort(sizes)[::n_req // 16][:16].tolist())
    rows = {k: [] for k in modes}
    keep = set(range(0, 200, 10))
    for j, n in enumerate(sizes):
        scj = scenes.lattice_container(rng, int(n), name=f"req{j}")
        if j not in pick:
            continue
        st = gpu_states(scj, 200, keep)
        for name, m in modes.items():
            rows[name] += _oracle_timed_steps(O, threads, scj, st, m)
    out["C4"] = {k: _cpu_row(r, "16 of the 12,000 requests (stratified by size), one at a "
                                "time, 200 steps (every 10th)") for k, r in rows.items()}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-table", action="store_true",
                    help="print the CPU baseline of every configuration and exit")
    ap.add_argument("--workload", default="column", choices=["column", "settling"])
    ap.add_argument("--cpu-budget-s", type=float, default=30.0)
    ap.add_argument("--ref-budget-s", type=float, default=150.0)
    ap.add_argument("--ref-tol-steps", type=int, default=2,
                    help="steps of the compacting column the reference arm times")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--max-iterations", type=int, default=None,
                    help="override the APGD iteration cap (profiling runs only)")
    ap.add_argument("--warm-start", default="positional", choices=["positional", "matched"],
                    help="warm-start semantics of the headline workload (positional is the "
                         "reference's; matched follows each (A, B) pair)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="precision of the headline workload (fp64 is the plain drop-in)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-scenes line")
    ap.add_argument("--no-column-at-tolerance", action="store_true",
                    help="skip the headline state stepped to the APGD tolerance")
    ap.add_argument("--tol-steps", type=int, default=10)
    ap.add_argument("--no-mixed-error", action="store_true",
                    help="skip the mixed-precision error report")
    ap.add_argument("--refine", type=int, default=500,
                    help="FP64 refinement iterations of the batched and served mixed-precision "
                         "solves (0: FP32 iterates alone)")
    ap.add_argument("--batch-scenes", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=100)
    ap.add_argument("--batch-timed", type=int, default=40)
    ap.add_argument("--plain-sample", type=int, default=16)
    ap.add_argument("--no-served", action="store_true", help="skip the served line")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--serve-steps", type=int, default=200)
    ap.add_argument("--serve-round", type=int, default=4)
    ap.add_argument("--serve-max-bodies", type=int, default=0,
                    help="resident-body limit of the server (0: none; the 4,096-scene and "
                         "150 GB limits still hold)")
    ap.add_argument("--serve-trace-s", type=float, default=5.0,
                    help="interval of the served line's backlog trace")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 0)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.cpu_table:
        print(json.dumps(run_cpu_table(args)), flush=True)
        return 0
    if args.impl == "reference":
        if rank != 0:
            return 0
        sc, desc = load_workload(args.workload)
        print(json.dumps(run_reference(args, sc, desc)), flush=True)
        return 0

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from dvide_b200 import _native as N
    sc, desc = load_workload(args.workload)
    if args.max_iterations is not None:
        sc.params["max_iterations"] = args.max_iterations
        desc += f" (maxIter overridden to {args.max_iterations})"
    if args.warm_start == "matched":
        sc.params["warm_start"] = 2
        desc += ", warm start matched by contact pair"
    prec = N.DV_PREC_MIXED if args.precision == "mixed" else N.DV_PREC_FP64
    if prec == N.DV_PREC_MIXED:
        desc = desc.replace("FP64", "mixed precision (FP32 iterates, FP64 sums and update)")
    g = N.NativeScene.from_scene(sc, precision=prec)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    g.set_stream(stream.cuda_stream)
    nb = sc.nb

    g.step(max(args.warmup, 3))
    g.history(clear=True)
    g.phase_times(reset=True)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # the e2e leg repeats exactly these steps: keep their starting state
    p_start, v_start = g.state()
    gamma_start = g.gamma()
    sampler = ClockSampler(local_rank)
    sampler.start()
    barrier()
    l0 = g.launches()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.step(args.steps)
    e1.record(stream)
    barrier()
    clocks = sampler.stop()
    launches = g.launches() - l0
    ms = e0.elapsed_time(e1)
    hist = g.history(clear=True)
    phases = g.phase_times(reset=True)
    contacts = sum(h["num_contacts"] for h in hist)
    t_local = ms / 1e3

    # end-to-end through the host-buffer API: state in from pinned memory, out every step
    p_host = torch.empty((nb, 3), dtype=torch.float64, pin_memory=True).numpy()
    v_host = torch.empty((nb, 3), dtype=torch.float64, pin_memory=True).numpy()
    p_host[:] = p_start
    v_host[:] = v_start
    g.set_gamma(gamma_start)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        g.set_state(p_host, v_host)
        g.step(1)
        g.state_into(p_host, v_host)
    barrier()
    t_e2e = time.perf_counter() - t0
    hist_e2e = g.history(clear=True)
    contacts_e2e = sum(h["num_contacts"] for h in hist_e2e)

    from dvide_b200 import replicas
    contacts_all, t_all = replicas.combine_timed_region(dist, contacts, t_local, device="cuda")
    contacts_e2e_all, t_e2e_all = replicas.combine_timed_region(dist, contacts_e2e, t_e2e,
                                                                device="cuda")

    if rank == 0:
        peak, peak_kind = _peaks()
        solve_ms = np.array([h["solve_ms"] for h in hist])
        step_ms = np.array([h["elapsed_ms"] for h in hist])
        ncs = np.array([h["num_contacts"] for h in hist])
        bts = np.array([h["backtracks"] for h in hist])
        sweeps = np.array([h["sweeps"] for h in hist])
        its = np.array([h["iterations"] for h in hist])
        nposs = np.array([h["num_possible"] for h in hist])
        bytes_per_launch = np.array([solve_bytes(c, nb, s, b) for c, s, b in zip(ncs, sweeps, bts)])
        own_bytes = np.array([solve_bytes_one_product(c, nb, s, b)
                              for c, s, b in zip(ncs, sweeps, bts)])
        achieved = float(bytes_per_launch.sum() / (solve_ms.sum() / 1e3) / 1e9)
        achieved_own = float(own_bytes.sum() / (solve_ms.sum() / 1e3) / 1e9)
        traffic = float(bytes_per_launch.mean() * TRAFFIC_PER_ALGORITHMIC_BYTE)
        dram_gbs = traffic / (solve_ms.mean() / 1e3) / 1e9
        tol = sc.params["tolerance"]
        line = {
            "metric": "contact-steps/s", "value": contacts_all / t_all, "unit": "contact-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": 1e3 * t_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == N.DV_PREC_FP64 else "f32+f64",
            "data": "synthetic (seeded scene, see config)",
            "config": {"workload": desc, "contacts_per_step": float(ncs.mean()),
                       "bodies": nb, "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (working set ~0.5 GB)",
                       "apgd_tolerance": tol, "apgd_max_iterations": int(sc.params["max_iterations"])},
            "convergence": {
                "iterations_mean": float(its.mean()), "backtracks_mean": float(bts.mean()),
                "residual_max": float(max(h["residual"] for h in hist)),
                "residual_last": hist[-1]["residual"],
                "steps_at_tolerance": f"{sum(1 for h in hist if h['residual'] < tol)}/{len(hist)}",
                "note": ("at rest every step reaches the iteration cap and reports its best "
                         "residual; column_at_tolerance is the same column while it compacts, "
                         "where every timed step reaches the tolerance")},
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                           "p99": float(np.percentile(step_ms, 99))},
            "apgd": {"iterations_mean": float(its.mean()), "sweeps_mean": float(sweeps.mean()),
                     "backtracks_mean": float(bts.mean()),
                     "residual_last": hist[-1]["residual"], "solve_ms_mean": float(solve_ms.mean()),
                     "collide_ms_mean": float(np.mean([h["collide_ms"] for h in hist])),
                     "phase_ms_total": {k: round(v[0], 3) for k, v in phases.items()},
                     "phase_us_mean": {k: round(1e3 * v[0] / v[1], 2) for k, v in phases.items()}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": traffic,
                         "kernel": "k_step_solve (persistent APGD + update)",
                         "peak_kind": peak_kind,
                         "bytes_per_launch": float(bytes_per_launch.mean()),
                         "bytes_model": "compulsory bytes, two Schur products per APGD iteration",
                         "achieved_one_product_model": achieved_own,
                         "frac_one_product_model": achieved_own / peak,
                         "dram_gbs": dram_gbs, "dram_frac": dram_gbs / peak},
            "e2e": {"value": contacts_e2e_all / t_e2e_all, "unit": "contact-steps/s",
                    "h2d_bytes_per_step": 2 * 24 * nb, "d2h_bytes_per_step": 2 * 24 * nb},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if world == 1 and not args.no_column_at_tolerance and args.workload == "column":
            line["column_at_tolerance"] = run_column_at_tolerance(args, N, torch, stream)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_sample(sc, args.cpu_budget_s)
        if world == 1 and not args.no_mixed_error:
            line["mixed_precision_error"] = run_mixed_error(N, stream)
        if world == 1 and not args.no_batched:
            line["batched"] = run_batched(args, N, torch, stream)
        if world == 1 and not args.no_served:
            line["served"] = run_served(args, N, stream)
        print(json.dumps(line), flush=True)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
