"""ctypes binding of libdvide_b200.so (the C ABI declared in include/dvide.h).

The shared library holds every CUDA kernel of the contact step; there is no
CPU fallback.  Loading fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdvide_b200.so")

DV_OK = 0
DV_PREC_FP64 = 0
DV_PREC_MIXED = 1
DV_SOLVER_APGD = 1
DV_SOLVER_PGJ = 5
DV_SOLVER_PGS = 6
STATUS = {0: "DV_OK", 1: "DV_ERR_ARG", 2: "DV_ERR_CUDA", 3: "DV_ERR_NAN", 4: "DV_ERR_NOCONV",
          5: "DV_ERR_OOM", 6: "DV_ERR_TIMEOUT", 7: "DV_ERR_UNSUPPORTED", 8: "DV_ERR_ABORTED"}

# Every entry point declared in include/dvide.h (checked by the CPU tests).
EXPORTS = [
    "dv_params_default", "dv_scene_create", "dv_scene_destroy", "dv_scene_set_stream",
    "dv_set_params", "dv_step", "dv_collide", "dv_apgd_solve", "dv_get_state", "dv_set_state",
    "dv_get_contact_force", "dv_get_num_contacts", "dv_get_contacts", "dv_get_gamma",
    "dv_set_gamma", "dv_add_bilateral_dof", "dv_get_bilateral_gamma", "dv_get_frames",
    "dv_get_schur_vector", "dv_get_step_vectors", "dv_ccp_violation", "dv_energies",
    "dv_contact_forces_per_collision", "dv_get_step_stats", "dv_status_string", "dv_last_error",
    "dv_scene_launch_count", "dv_get_step_history", "dv_clear_step_history",
    "dv_get_phase_times", "dv_ccp_violation_noalloc", "dv_selftest_bounded_waits",
    "dv_batch_create", "dv_batch_destroy", "dv_batch_set_stream", "dv_batch_step",
    "dv_batch_num_scenes", "dv_batch_get_state", "dv_batch_set_state", "dv_batch_scene_stats",
    "dv_batch_step_history", "dv_batch_get_gamma", "dv_batch_ccp_violation",
    "dv_batch_set_launch", "dv_batch_get_launch", "dv_batch_set_graph", "dv_batch_autotune",
    "dv_batch_launch_count",
    "dv_server_default_config", "dv_server_create", "dv_server_destroy", "dv_server_set_stream",
    "dv_server_clock", "dv_server_submit", "dv_server_round", "dv_server_poll",
    "dv_server_result_state", "dv_server_get_stats",
]


class DvError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = f"{STATUS.get(status, status)}"
        if what:
            msg += f" in {what}"
        try:
            detail = lib().dv_last_error().decode()
            if detail:
                msg += f": {detail}"
        except Exception:  # pragma: no cover - library not loadable
            pass
        super().__init__(msg)


class BodyDesc(C.Structure):
    _fields_ = [("pos", C.c_double * 3), ("vel", C.c_double * 3), ("mass", C.c_double),
                ("geom", C.c_double * 3), ("fixed", C.c_int32), ("family", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("h", C.c_double), ("mu", C.c_double), ("gravity", C.c_double * 3),
                ("envelope", C.c_double), ("tolerance", C.c_double),
                ("max_iterations", C.c_int32), ("warm_start", C.c_int32), ("solver", C.c_int32),
                ("precision", C.c_int32), ("max_backtracks", C.c_int32), ("verbose", C.c_int32),
                ("fp64_narrowphase", C.c_int32), ("anti_relaxation", C.c_int32),
                ("refine_iterations", C.c_int32)]


class StepStats(C.Structure):
    _fields_ = [("num_contacts", C.c_int32), ("num_possible", C.c_int32),
                ("iterations", C.c_int32), ("backtracks", C.c_int32), ("residual", C.c_double),
                ("objective", C.c_double), ("elapsed_ms", C.c_double), ("time", C.c_double),
                ("time_index", C.c_int32), ("status", C.c_int32), ("collide_ms", C.c_double),
                ("solve_ms", C.c_double), ("sweeps", C.c_int32),
                ("refine_iterations", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SceneStats(C.Structure):
    _fields_ = [("num_contacts", C.c_int32), ("num_possible", C.c_int32),
                ("iterations", C.c_int32), ("backtracks", C.c_int32), ("residual", C.c_double),
                ("objective", C.c_double), ("status", C.c_int32), ("sweeps", C.c_int32),
                ("refine_iterations", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneCandidate(C.Structure):
    _fields_ = [("grid", C.c_int32), ("chunk", C.c_int32), ("contiguous", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("ms_per_step", C.c_float)]


class TuneReport(C.Structure):
    _fields_ = [("num_candidates", C.c_int32), ("best", C.c_int32), ("identical", C.c_int32),
                ("steps_per_trial", C.c_int32), ("cand", TuneCandidate * 16)]

    def as_dict(self):
        return {"best": self.best, "identical": bool(self.identical),
                "steps_per_trial": self.steps_per_trial,
                "candidates": [{"grid": c.grid, "chunk": c.chunk, "contiguous": c.contiguous,
                                "blocks_per_sm": c.blocks_per_sm, "ms_per_step": c.ms_per_step}
                               for c in self.cand[:self.num_candidates]]}


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_double), ("max_active", C.c_int32),
                ("steps_per_round", C.c_int32), ("precision", C.c_int32), ("use_graph", C.c_int32),
                ("keep_states", C.c_int32), ("max_resident_bodies", C.c_int32)]


class RequestResult(C.Structure):
    _fields_ = [("id", C.c_int64), ("nb", C.c_int32), ("nsteps", C.c_int32),
                ("status", C.c_int32), ("rounds", C.c_int32), ("solves", C.c_int32),
                ("solves_at_tolerance", C.c_int32), ("t_submit", C.c_double),
                ("t_admit", C.c_double), ("t_done", C.c_double), ("contact_steps", C.c_double),
                ("step_ms_mean", C.c_double), ("step_ms_p50", C.c_double),
                ("step_ms_p99", C.c_double), ("bytes", C.c_double),
                ("iterations", C.c_double), ("iteration_contacts", C.c_double),
                ("refine_iterations", C.c_double), ("refine_iteration_contacts", C.c_double),
                ("backtracks", C.c_double), ("backtrack_contacts", C.c_double),
                ("refined_solves", C.c_double), ("refined_contacts", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("pending", C.c_int64), ("active", C.c_int64), ("rounds", C.c_int64),
                ("reconfigures", C.c_int64), ("steps", C.c_int64), ("bytes_in_use", C.c_double),
                ("contact_steps", C.c_double), ("device_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# numpy layout of dv_body_desc (88 bytes, no padding)
BODY_DTYPE = np.dtype([("pos", "<f8", 3), ("vel", "<f8", 3), ("mass", "<f8"), ("geom", "<f8", 3),
                       ("fixed", "<i4"), ("family", "<i4")])
assert BODY_DTYPE.itemsize == C.sizeof(BodyDesc)

_lib = None


def lib():
    """Loads libdvide_b200.so; raises if it is missing (no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built; run dvide_b200.build.build()")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip, up = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_uint32)
    sig = {
        "dv_params_default": [C.POINTER(Params)],
        "dv_scene_create": [C.POINTER(BodyDesc), C.c_int32, C.POINTER(Params), C.POINTER(vp)],
        "dv_scene_destroy": [vp],
        "dv_scene_set_stream": [vp, vp],
        "dv_set_params": [vp, C.POINTER(Params)],
        "dv_step": [vp, C.c_int32],
        "dv_apgd_solve": [vp],
        "dv_collide": [vp],
        "dv_get_state": [vp, dp, dp],
        "dv_set_state": [vp, dp, dp],
        "dv_get_contact_force": [vp, dp],
        "dv_get_num_contacts": [vp, ip, ip],
        "dv_get_contacts": [vp, up, up, dp, dp],
        "dv_get_gamma": [vp, dp, C.c_int32, ip],
        "dv_set_gamma": [vp, dp, C.c_int32],
        "dv_add_bilateral_dof": [vp, C.c_int32, C.c_int32, C.c_double, C.c_double],
        "dv_get_step_vectors": [vp, dp, dp, dp],
        "dv_get_bilateral_gamma": [vp, dp, C.c_int32, ip],
        "dv_get_frames": [vp, dp],
        "dv_get_schur_vector": [vp, dp],
        "dv_ccp_violation": [vp, dp],
        "dv_energies": [vp, dp, dp],
        "dv_contact_forces_per_collision": [vp, dp, dp],
        "dv_get_step_stats": [vp, C.POINTER(StepStats)],
        "dv_get_step_history": [vp, C.POINTER(StepStats), C.c_int32, ip],
        "dv_clear_step_history": [vp],
        "dv_get_phase_times": [vp, dp, C.POINTER(C.c_int64), C.c_int32],
        "dv_batch_create": [C.POINTER(BodyDesc), ip, C.c_int32, C.POINTER(Params), C.c_int32,
                            C.POINTER(vp)],
        "dv_batch_destroy": [vp],
        "dv_batch_set_stream": [vp, vp],
        "dv_batch_step": [vp, C.c_int32],
        "dv_batch_num_scenes": [vp, ip, ip],
        "dv_batch_get_state": [vp, C.c_int32, dp, dp],
        "dv_batch_set_state": [vp, C.c_int32, dp, dp],
        "dv_batch_scene_stats": [vp, C.POINTER(SceneStats)],
        "dv_batch_step_history": [vp, C.POINTER(SceneStats), C.POINTER(C.c_float), C.c_int32, ip],
        "dv_batch_get_gamma": [vp, C.c_int32, dp, C.c_int32, ip],
        "dv_batch_ccp_violation": [vp, C.c_int32, dp],
        "dv_batch_set_launch": [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32],
        "dv_batch_get_launch": [vp, ip, ip, ip, ip, ip],
        "dv_batch_set_graph": [vp, C.c_int32],
        "dv_batch_autotune": [vp, C.c_int32, C.POINTER(TuneReport)],
        "dv_server_default_config": [C.POINTER(ServerConfig)],
        "dv_server_create": [C.POINTER(ServerConfig), C.POINTER(vp)],
        "dv_server_destroy": [vp],
        "dv_server_set_stream": [vp, vp],
        "dv_server_submit": [vp, C.POINTER(BodyDesc), C.c_int32, C.POINTER(Params), C.c_int32,
                             C.POINTER(C.c_int64)],
        "dv_server_round": [vp, ip],
        "dv_server_poll": [vp, C.POINTER(RequestResult), C.c_int32, ip],
        "dv_server_result_state": [vp, C.c_int64, dp, dp],
        "dv_server_get_stats": [vp, C.POINTER(ServerStats)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.dv_status_string.argtypes = [C.c_int]
    L.dv_status_string.restype = C.c_char_p
    L.dv_last_error.argtypes = []
    L.dv_last_error.restype = C.c_char_p
    L.dv_ccp_violation_noalloc.argtypes = [C.c_int32, C.c_int32, vp, vp, vp, vp, vp, C.c_double,
                                           C.c_double, vp, vp]
    L.dv_ccp_violation_noalloc.restype = C.c_int
    L.dv_scene_launch_count.argtypes = [vp]
    L.dv_scene_launch_count.restype = C.c_int64
    L.dv_batch_launch_count.argtypes = [vp]
    L.dv_batch_launch_count.restype = C.c_int64
    L.dv_server_clock.argtypes = [vp]
    L.dv_server_clock.restype = C.c_double
    _lib = L
    return L


def check(status, what=""):
    if status != DV_OK:
        raise DvError(status, what)


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def uptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def make_params(p: dict, precision=DV_PREC_FP64) -> Params:
    o = Params()
    lib().dv_params_default(C.byref(o))
    o.h = float(p.get("h", o.h))
    o.mu = float(p.get("mu", o.mu))
    if "gravity" in p:
        o.gravity[:] = [float(x) for x in p["gravity"]]
    o.envelope = float(p.get("envelope", o.envelope))
    o.tolerance = float(p.get("tolerance", o.tolerance))
    o.max_iterations = int(p.get("max_iterations", o.max_iterations))
    o.warm_start = int(p.get("warm_start", o.warm_start))
    o.solver = int(p.get("solver", o.solver))
    o.max_backtracks = int(p.get("max_backtracks", o.max_backtracks))
    o.precision = int(p.get("precision", precision))
    o.verbose = int(p.get("verbose", 0))
    o.fp64_narrowphase = int(p.get("fp64_narrowphase", 0))
    o.anti_relaxation = int(p.get("anti_relaxation", 0))
    o.refine_iterations = int(p.get("refine_iterations", 0))
    return o


def body_records(pos, vel, mass, geom, fixed, family):
    """dv_body_desc records as a numpy structured array."""
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    nb = pos.shape[0]
    rec = np.zeros(max(nb, 1), dtype=BODY_DTYPE)
    if nb:
        rec["pos"][:nb] = pos
        rec["vel"][:nb] = np.asarray(vel, dtype=np.float64).reshape(-1, 3)
        rec["mass"][:nb] = np.asarray(mass, dtype=np.float64)
        rec["geom"][:nb] = np.asarray(geom, dtype=np.float64).reshape(-1, 3)
        rec["fixed"][:nb] = np.asarray(fixed, dtype=np.int32)
        rec["family"][:nb] = np.asarray(family, dtype=np.int32)
    return rec, nb


def body_array(pos, vel, mass, geom, fixed, family):
    rec, nb = body_records(pos, vel, mass, geom, fixed, family)
    return rec.ctypes.data_as(C.POINTER(BodyDesc)), nb, rec


class NativeScene:
    """One device-resident scene (dv_scene*) driven through the C ABI."""

    def __init__(self, pos, vel, mass, geom, fixed, family, params: dict,
                 precision=DV_PREC_FP64):
        L = lib()
        arr, nb, self._rec = body_array(pos, vel, mass, geom, fixed, family)
        self.nb = nb
        self.params = make_params(params, precision)
        h = C.c_void_p()
        check(L.dv_scene_create(arr, nb, C.byref(self.params), C.byref(h)), "dv_scene_create")
        self.h = h

    @classmethod
    def from_scene(cls, scene, precision=DV_PREC_FP64, **overrides):
        p = dict(scene.params)
        p.update(overrides)
        g = cls(scene.pos, scene.vel, scene.mass, scene.geom, scene.fixed, scene.family, p,
                precision)
        if getattr(scene, "gamma", None) is not None:
            g.set_gamma(scene.gamma)
        for row in getattr(scene, "bilateral", None) or ():
            g.add_bilateral(*row)
        return g

    def close(self):
        if getattr(self, "h", None):
            lib().dv_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, **kw):
        for k, v in kw.items():
            if k == "gravity":
                self.params.gravity[:] = list(v)
            else:
                setattr(self.params, k, v)
        check(lib().dv_set_params(self.h, C.byref(self.params)), "dv_set_params")

    def set_stream(self, stream_ptr):
        check(lib().dv_scene_set_stream(self.h, C.c_void_p(stream_ptr)), "dv_scene_set_stream")

    def step(self, n=1, raise_on_error=True):
        st = lib().dv_step(self.h, int(n))
        if raise_on_error:
            check(st, "dv_step")
        return st

    def collide(self):
        check(lib().dv_collide(self.h), "dv_collide")

    def solve(self, raise_on_error=True):
        """The scene solver's solve() alone (dv_apgd_solve): no update."""
        st = lib().dv_apgd_solve(self.h)
        if raise_on_error:
            check(st, "dv_apgd_solve")
        return st

    def state(self):
        p = np.zeros((self.nb, 3))
        v = np.zeros((self.nb, 3))
        check(lib().dv_get_state(self.h, dptr(p), dptr(v)), "dv_get_state")
        return p, v

    def state_into(self, p, v):
        """Copies positions and velocities into caller arrays (e.g. pinned)."""
        check(lib().dv_get_state(self.h, dptr(p), dptr(v)), "dv_get_state")

    def set_state(self, p=None, v=None):
        pp = np.ascontiguousarray(p, dtype=np.float64) if p is not None else None
        vv = np.ascontiguousarray(v, dtype=np.float64) if v is not None else None
        check(lib().dv_set_state(self.h, dptr(pp) if pp is not None else None,
                                 dptr(vv) if vv is not None else None), "dv_set_state")

    def fcontact(self):
        f = np.zeros((self.nb, 3))
        check(lib().dv_get_contact_force(self.h, dptr(f)), "dv_get_contact_force")
        return f

    def num_contacts(self):
        nc = C.c_int32()
        np_ = C.c_int32()
        check(lib().dv_get_num_contacts(self.h, C.byref(nc), C.byref(np_)))
        return nc.value, np_.value

    def contacts(self):
        nc, _ = self.num_contacts()
        a = np.zeros(nc, dtype=np.uint32)
        b = np.zeros(nc, dtype=np.uint32)
        nP = np.zeros((nc, 4))
        loc = np.zeros((nc, 3))
        if nc:
            check(lib().dv_get_contacts(self.h, uptr(a), uptr(b), dptr(nP), dptr(loc)))
        return a, b, nP, loc

    def frames(self):
        nc, _ = self.num_contacts()
        F = np.zeros((nc, 9))
        if nc:
            check(lib().dv_get_frames(self.h, dptr(F)))
        return F

    def r(self):
        nc, _ = self.num_contacts()
        r = np.zeros((nc, 3))
        if nc:
            check(lib().dv_get_schur_vector(self.h, dptr(r)))
        return r

    def gamma(self):
        n = C.c_int32()
        check(lib().dv_get_gamma(self.h, None, 0, C.byref(n)))
        g = np.zeros((n.value, 3))
        if n.value:
            check(lib().dv_get_gamma(self.h, dptr(g), n.value, C.byref(n)))
        return g

    def set_gamma(self, g):
        g = np.ascontiguousarray(g, dtype=np.float64).reshape(-1, 3)
        check(lib().dv_set_gamma(self.h, dptr(g), g.shape[0]), "dv_set_gamma")

    def add_bilateral(self, dof_a, dof_b=-1, velocity=0.0, start_time=0.0):
        """System::addBilateralConstraintDOF (before the first step)."""
        check(lib().dv_add_bilateral_dof(self.h, int(dof_a), int(dof_b), float(velocity),
                                         float(start_time)), "dv_add_bilateral_dof")

    def bilateral_gamma(self):
        n = C.c_int32()
        check(lib().dv_get_bilateral_gamma(self.h, None, 0, C.byref(n)))
        g = np.zeros(n.value)
        if n.value:
            check(lib().dv_get_bilateral_gamma(self.h, dptr(g), n.value, C.byref(n)))
        return g

    def step_vectors(self):
        """r, b (bilateral rows first, then 3 per contact) and k (3 per body)
        of the last step (System::r_d, b_d, k_d)."""
        n = 3 * self.num_contacts()[0] + len(self.bilateral_gamma())
        r, b, k = np.zeros(n), np.zeros(n), np.zeros(3 * self.nb)
        check(lib().dv_get_step_vectors(self.h, dptr(r), dptr(b), dptr(k)))
        return r, b, k

    def ccp_violation(self):
        o = np.zeros(4)
        check(lib().dv_ccp_violation(self.h, dptr(o)))
        return o

    def energies(self):
        k = C.c_double()
        p = C.c_double()
        check(lib().dv_energies(self.h, C.byref(k), C.byref(p)))
        return k.value, p.value

    def contact_forces(self):
        nc, _ = self.num_contacts()
        n = np.zeros((nc, 3))
        f = np.zeros((nc, 3))
        if nc:
            check(lib().dv_contact_forces_per_collision(self.h, dptr(n), dptr(f)))
        return n, f

    def stats(self):
        s = StepStats()
        lib().dv_get_step_stats(self.h, C.byref(s))
        return s.as_dict()

    def history(self, clear=False):
        n = C.c_int32()
        lib().dv_get_step_history(self.h, None, 0, C.byref(n))
        arr = (StepStats * max(n.value, 1))()
        lib().dv_get_step_history(self.h, arr, n.value, C.byref(n))
        out = [arr[i].as_dict() for i in range(n.value)]
        if clear:
            lib().dv_clear_step_history(self.h)
        return out

    PHASES = ("setup", "step", "backtrack", "body", "product", "final", "unused6", "unused7")

    def phase_times(self, reset=False):
        ns = np.zeros(8)
        cnt = np.zeros(8, dtype=np.int64)
        check(lib().dv_get_phase_times(self.h, dptr(ns), cnt.ctypes.data_as(C.POINTER(C.c_int64)),
                                       int(reset)))
        return {name: (float(ns[i]) / 1e6, int(cnt[i])) for i, name in enumerate(self.PHASES)
                if cnt[i]}

    def launches(self):
        return int(lib().dv_scene_launch_count(self.h))


def selftest_bounded_waits(limit_ms=50):
    """Runs the solve kernels' bounded waits against conditions that never come
    true (dv_selftest_bounded_waits); returns (barrier_timed_out,
    copy_timed_out, error_bits)."""
    b, c, e = C.c_int32(), C.c_int32(), C.c_uint32()
    check(lib().dv_selftest_bounded_waits(int(limit_ms), C.byref(b), C.byref(c), C.byref(e)),
          "dv_selftest_bounded_waits")
    return b.value, c.value, e.value


class NativeBatch:
    """Many scenes stepped together (dv_batch*): one collision pipeline and one
    persistent solve kernel per step for all of them."""

    def __init__(self, scenes_list, precision=DV_PREC_FP64, **overrides):
        L = lib()
        recs = []
        counts = []
        params = (Params * len(scenes_list))()
        for i, sc in enumerate(scenes_list):
            rec, nb = body_records(sc.pos, sc.vel, sc.mass, sc.geom, sc.fixed, sc.family)
            recs.append(rec[:nb])
            counts.append(nb)
            p = dict(sc.params)
            p.update(overrides)
            params[i] = make_params(p, precision)
        self._rec = np.concatenate(recs)
        self.counts = np.asarray(counts, dtype=np.int32)
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        self.nscenes = len(scenes_list)
        self.nb = int(self.offsets[-1])
        h = C.c_void_p()
        check(L.dv_batch_create(self._rec.ctypes.data_as(C.POINTER(BodyDesc)),
                                self.counts.ctypes.data_as(C.POINTER(C.c_int32)), self.nscenes,
                                params, int(precision), C.byref(h)), "dv_batch_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().dv_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        check(lib().dv_batch_step(self.h, int(n)), "dv_batch_step")

    def set_stream(self, stream_ptr):
        check(lib().dv_batch_set_stream(self.h, C.c_void_p(stream_ptr)), "dv_batch_set_stream")

    def state(self, scene=-1):
        n = self.nb if scene < 0 else int(self.counts[scene])
        p = np.zeros((n, 3))
        v = np.zeros((n, 3))
        check(lib().dv_batch_get_state(self.h, int(scene), dptr(p), dptr(v)), "dv_batch_get_state")
        return p, v

    def state_into(self, p, v):
        check(lib().dv_batch_get_state(self.h, -1, dptr(p), dptr(v)), "dv_batch_get_state")

    def set_state(self, scene, p=None, v=None):
        pp = np.ascontiguousarray(p, dtype=np.float64) if p is not None else None
        vv = np.ascontiguousarray(v, dtype=np.float64) if v is not None else None
        check(lib().dv_batch_set_state(self.h, int(scene), dptr(pp) if pp is not None else None,
                                       dptr(vv) if vv is not None else None), "dv_batch_set_state")

    def scene_stats(self):
        arr = (SceneStats * self.nscenes)()
        check(lib().dv_batch_scene_stats(self.h, arr), "dv_batch_scene_stats")
        return [arr[i].as_dict() for i in range(self.nscenes)]

    def history(self):
        n = C.c_int32()
        check(lib().dv_batch_step_history(self.h, None, None, 0, C.byref(n)))
        steps = n.value
        arr = (SceneStats * max(steps * self.nscenes, 1))()
        ms = (C.c_float * max(steps, 1))()
        check(lib().dv_batch_step_history(self.h, arr, ms, steps, C.byref(n)))
        out = [[arr[i * self.nscenes + s].as_dict() for s in range(self.nscenes)]
               for i in range(steps)]
        return out, [float(ms[i]) for i in range(steps)]

    def gamma(self, scene):
        n = C.c_int32()
        check(lib().dv_batch_get_gamma(self.h, int(scene), None, 0, C.byref(n)))
        g = np.zeros((max(n.value, 0), 3))
        if n.value:
            check(lib().dv_batch_get_gamma(self.h, int(scene), dptr(g), n.value, C.byref(n)))
        return g

    def ccp_violation(self, scene):
        o = np.zeros(4)
        check(lib().dv_batch_ccp_violation(self.h, int(scene), dptr(o)))
        return o

    def set_launch(self, grid=0, chunk=1, contiguous=0, blocks_per_sm=2):
        check(lib().dv_batch_set_launch(self.h, int(grid), int(chunk), int(contiguous),
                                        int(blocks_per_sm)))

    def launch(self):
        g, c, k, bps, m = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().dv_batch_get_launch(self.h, C.byref(g), C.byref(c), C.byref(k), C.byref(bps),
                                        C.byref(m)))
        return {"grid": g.value, "chunk": c.value, "contiguous": k.value,
                "blocks_per_sm": bps.value, "max_grid": m.value}

    def set_graph(self, on=True):
        return lib().dv_batch_set_graph(self.h, int(bool(on)))

    def autotune(self, steps_per_trial=2):
        rep = TuneReport()
        st = lib().dv_batch_autotune(self.h, int(steps_per_trial), C.byref(rep))
        out = rep.as_dict()
        out["status"] = st
        return out

    def launches(self):
        return int(lib().dv_batch_launch_count(self.h))


class NativeServer:
    """Continuous-batching server (dv_server*): requests are admitted as slots and
    the HBM budget allow, resident scenes step together, finished ones leave."""

    def __init__(self, precision=DV_PREC_MIXED, hbm_budget_bytes=150e9, max_active=4096,
                 steps_per_round=4, use_graph=True, keep_states=True, max_resident_bodies=0):
        L = lib()
        cfg = ServerConfig()
        check(L.dv_server_default_config(C.byref(cfg)))
        cfg.hbm_budget_bytes = float(hbm_budget_bytes)
        cfg.max_active = int(max_active)
        cfg.steps_per_round = int(steps_per_round)
        cfg.precision = int(precision)
        cfg.use_graph = int(bool(use_graph))
        cfg.keep_states = int(bool(keep_states))
        cfg.max_resident_bodies = int(max_resident_bodies)
        self.cfg = cfg
        h = C.c_void_p()
        check(L.dv_server_create(C.byref(cfg), C.byref(h)), "dv_server_create")
        self.h = h
        self.sizes = {}

    def close(self):
        if getattr(self, "h", None):
            lib().dv_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        check(lib().dv_server_set_stream(self.h, C.c_void_p(stream_ptr)))

    def clock(self):
        return float(lib().dv_server_clock(self.h))

    def submit(self, scene, nsteps, **overrides):
        rec, nb = body_records(scene.pos, scene.vel, scene.mass, scene.geom, scene.fixed,
                               scene.family)
        p = dict(scene.params)
        p.update(overrides)
        prm = make_params(p, self.cfg.precision)
        rid = C.c_int64()
        check(lib().dv_server_submit(self.h, rec.ctypes.data_as(C.POINTER(BodyDesc)), nb,
                                     C.byref(prm), int(nsteps), C.byref(rid)), "dv_server_submit")
        self.sizes[rid.value] = nb
        return rid.value

    def round(self):
        busy = C.c_int32()
        check(lib().dv_server_round(self.h, C.byref(busy)), "dv_server_round")
        return bool(busy.value)

    def poll(self, cap=4096):
        arr = (RequestResult * cap)()
        n = C.c_int32()
        check(lib().dv_server_poll(self.h, arr, cap, C.byref(n)))
        return [arr[i].as_dict() for i in range(n.value)]

    def result_state(self, rid):
        nb = self.sizes[rid]
        p = np.zeros((nb, 3))
        v = np.zeros((nb, 3))
        check(lib().dv_server_result_state(self.h, int(rid), dptr(p), dptr(v)))
        return p, v

    def stats(self):
        st = ServerStats()
        check(lib().dv_server_get_stats(self.h, C.byref(st)))
        return st.as_dict()

