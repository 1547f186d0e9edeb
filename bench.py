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


# DRAM bytes per algorithmic byte of the solve kernel, measured with ncu
# (dram__bytes_read.sum + dram__bytes_write.sum = 6.350 GB) on a 30-iteration
# launch on this workload (11.415 GB algorithmic); the full launch is scaled by it.
TRAFFIC_PER_ALGORITHMIC_BYTE = 6.244004 / 11.415179


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


def run_reference(args, sc, desc):
    """The reference's algorithm on the host cores (oracle/), same state and config."""
    from oracle import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    o = O.OracleScene(sc, threads=threads)
    budget = args.ref_budget_s
    warm = 1 if args.warmup > 0 else 0
    t0 = time.perf_counter()
    o.step(warm)
    t_warm = time.perf_counter() - t0
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
    sample = (f"{done} of {args.steps} full time steps after {warm} warm-up step "
              f"({t_warm:.1f} s), {threads} OpenMP threads, oracle port of APGD/System")
    return {"metric": "contact-steps/s", "value": value, "unit": "contact-steps/s",
            "impl": "reference", "n_gpus": 0, "steps": done, "warmup": warm,
            "ms_per_step": 1e3 * dt / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc},
            "cpu_baseline": {"value": value, "unit": "contact-steps/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "contact-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def cpu_baseline_sample(sc, budget_s):
    from oracle import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    o = O.OracleScene(sc, threads=threads)
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
                      f"start, {dt:.1f} s"}


def run_mixed_error(N, stream, steps=500, every=10):
    """Mixed precision (FP32 iterates, FP64 sums and update) against FP64 on the
    1,000-sphere settling box (h 1e-3, at most 1000 iterations, warm start):
    every `every`-th of `steps` steps, the mixed solve starts from the FP64
    run's state and warm start and both take one step; relative 2-norm errors
    of gamma and v, the largest velocity difference, and both residuals.  At
    the benchmark tolerance 1e-4 the two solves stop at different iterates, so
    the difference includes the solver tolerance; at 1e-6 it is the precision.
    The FP64 path gives the oracle's results bit for bit
    (tests/test_gpu_parity.py)."""
    from dvide_b200 import scenes

    def rel(a, b):
        n = float(np.linalg.norm(b))
        d = float(np.linalg.norm(a - b))
        return d / n if n > 0 else d

    out = {"workload": (f"settling_box 1000 spheres, every {every}th of {steps} steps "
                        f"(teacher-forced from the FP64 run), h 1e-3, maxIter 1000")}
    for tol in (1e-4, 1e-6):
        sc = scenes.settling_box(tolerance=tol)
        f = N.NativeScene.from_scene(sc)
        m = N.NativeScene.from_scene(sc, precision=N.DV_PREC_MIXED)
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
            rows.append((rel(m.gamma(), f.gamma()), rel(vm, vf), float(np.abs(vm - vf).max()),
                         sf["residual"], sm["residual"], sf["iterations"], sm["iterations"]))
        f.close()
        m.close()
        if not rows:
            continue
        a = np.array(rows)
        out[f"tolerance_{tol:g}"] = {
            "steps_compared": len(rows),
            "gamma_rel_err": {"max": float(a[:, 0].max()), "median": float(np.median(a[:, 0]))},
            "v_rel_err": {"max": float(a[:, 1].max()), "median": float(np.median(a[:, 1]))},
            "v_abs_err_max_m_per_s": float(a[:, 2].max()),
            "residual_fp64_max": float(a[:, 3].max()),
            "residual_mixed_max": float(a[:, 4].max()),
            "iterations_mean": {"fp64": float(a[:, 5].mean()), "mixed": float(a[:, 6].mean())},
        }
    return out


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
    b = N.NativeBatch(scs, precision=N.DV_PREC_MIXED)
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
                     f"{total_steps} timed (h 1e-3), mixed precision, per-scene convergence"),
        "value": batched, "unit": "contact-steps/s", "ms_per_step": ms / timed,
        "contacts_per_step": contacts / timed,
        "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                       "p99": float(np.percentile(step_ms, 99))},
        "scene_iterations_mean": float(np.mean(iters)) if iters else 0.0,
        "scene_solves_converged": f"{conv}/{len(res)}",
        "graph": graph, "autotune": {"best": tune["candidates"][tune["best"]],
                                      "identical": tune["identical"]},
        "gpu_launches": int(launches),
        "plain_fp64_one_at_a_time": {
            "value": plain, "unit": "contact-steps/s",
            "sample": f"{len(sample)} of {len(scs)} scenes (every {len(scs) // len(sample)}th by "
                      f"size), same steps, device time"},
        "speedup_vs_plain": (batched / plain) if plain else None,
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
    reqs = [scenes.lattice_container(rng, int(n), name=f"req{i}") for i, n in enumerate(sizes)]
    srv = N.NativeServer(precision=N.DV_PREC_MIXED, hbm_budget_bytes=150e9,
                         steps_per_round=args.serve_round, keep_states=False)
    srv.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    i = 0
    results = []
    busy = False
    while i < n_req or busy:
        now = time.perf_counter() - t0
        while i < n_req and arrive[i] <= now:
            srv.submit(reqs[i], args.serve_steps)
            i += 1
        if not busy and i < n_req and arrive[i] > now:
            time.sleep(min(arrive[i] - now, 0.01))
            busy = srv.stats()["active"] > 0 or srv.stats()["pending"] > 0
            continue
        busy = srv.round()
        results += srv.poll()
    wall = time.perf_counter() - t0
    results += srv.poll()
    st = srv.stats()
    srv.close()
    lat = np.array([r["t_done"] - r["t_submit"] for r in results])
    step_p50 = np.array([r["step_ms_p50"] for r in results])
    step_p99 = np.array([r["step_ms_p99"] for r in results])
    contact_steps = st["contact_steps"]
    # plain FP64 one request at a time on a stratified sample
    order = np.argsort(sizes)
    pick = order[::max(1, n_req // args.plain_sample)]
    p_cs, p_ms = 0.0, 0.0
    for j in pick:
        g = N.NativeScene.from_scene(reqs[j])
        g.set_stream(stream.cuda_stream)
        g.step(args.serve_steps)
        h = g.history(clear=True)
        p_cs += sum(x["num_contacts"] for x in h)
        p_ms += sum(x["elapsed_ms"] for x in h)
        g.close()
    plain = p_cs / (p_ms / 1e3) if p_ms > 0 else None
    served = contact_steps / wall
    return {
        "workload": (f"{n_req} requests, Poisson {args.serve_rate}/s for {args.serve_seconds} s, "
                     f"{args.serve_steps} steps each (h 1e-3), spheres log-uniform [500, 50000], "
                     f"mixed precision, 150 GB budget"),
        "value": served, "unit": "contact-steps/s (wall clock, arrivals included)",
        "device_contact_steps_per_s": contact_steps / (st["device_ms"] / 1e3),
        "wall_s": wall, "completed": int(st["completed"]), "rounds": int(st["rounds"]),
        "layout_changes": int(st["reconfigures"]),
        "time_per_step_ms": {"p50": float(np.percentile(step_p50, 50)),
                             "p99": float(np.percentile(step_p99, 99))},
        "completion_latency_s": {"p50": float(np.percentile(lat, 50)),
                                 "p99": float(np.percentile(lat, 99))},
        "plain_fp64_one_at_a_time": {
            "value": plain, "unit": "contact-steps/s (device time)",
            "sample": f"{len(pick)} of {n_req} requests (every {max(1, n_req // args.plain_sample)}th "
                      f"by size)"},
        "speedup_vs_plain": (served / plain) if plain else None,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="column", choices=["column", "settling"])
    ap.add_argument("--cpu-budget-s", type=float, default=30.0)
    ap.add_argument("--ref-budget-s", type=float, default=150.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--max-iterations", type=int, default=None,
                    help="override the APGD iteration cap (profiling runs only)")
    ap.add_argument("--warm-start", default="positional", choices=["positional", "matched"],
                    help="warm-start semantics of the headline workload (positional is the "
                         "reference's; matched follows each (A, B) pair)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="precision of the headline workload (fp64 is the plain drop-in)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-scenes line")
    ap.add_argument("--no-mixed-error", action="store_true",
                    help="skip the mixed-precision error report")
    ap.add_argument("--batch-scenes", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=100)
    ap.add_argument("--batch-timed", type=int, default=40)
    ap.add_argument("--plain-sample", type=int, default=16)
    ap.add_argument("--no-served", action="store_true", help="skip the served line")
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--serve-steps", type=int, default=200)
    ap.add_argument("--serve-round", type=int, default=4)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 0)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

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
        achieved = float(bytes_per_launch.sum() / (solve_ms.sum() / 1e3) / 1e9)
        line = {
            "metric": "contact-steps/s", "value": contacts_all / t_all, "unit": "contact-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": 1e3 * t_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == N.DV_PREC_FP64 else "f32+f64",
            "data": "synthetic (seeded scene, see config)",
            "config": {"workload": desc, "contacts_per_step": float(ncs.mean()),
                       "bodies": nb, "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (working set ~0.5 GB)"},
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
                         "traffic": float(bytes_per_launch.mean() * TRAFFIC_PER_ALGORITHMIC_BYTE),
                         "kernel": "k_step_solve (persistent APGD + update)",
                         "peak_kind": peak_kind,
                         "bytes_per_launch": float(bytes_per_launch.mean())},
            "e2e": {"value": contacts_e2e_all / t_e2e_all, "unit": "contact-steps/s",
                    "h2d_bytes_per_step": 2 * 24 * nb, "d2h_bytes_per_step": 2 * 24 * nb},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
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
