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
STATUS = {0: "DV_OK", 1: "DV_ERR_ARG", 2: "DV_ERR_CUDA", 3: "DV_ERR_NAN", 4: "DV_ERR_NOCONV",
          5: "DV_ERR_OOM", 6: "DV_ERR_TIMEOUT", 7: "DV_ERR_UNSUPPORTED", 8: "DV_ERR_ABORTED"}

# Every entry point declared in include/dvide.h (checked by the CPU tests).
EXPORTS = [
    "dv_params_default", "dv_scene_create", "dv_scene_destroy", "dv_scene_set_stream",
    "dv_set_params", "dv_step", "dv_collide", "dv_get_state", "dv_set_state",
    "dv_get_contact_force", "dv_get_num_contacts", "dv_get_contacts", "dv_get_gamma",
    "dv_set_gamma", "dv_get_frames", "dv_get_schur_vector", "dv_ccp_violation", "dv_energies",
    "dv_contact_forces_per_collision", "dv_get_step_stats", "dv_status_string", "dv_last_error",
    "dv_scene_launch_count", "dv_get_step_history", "dv_clear_step_history",
    "dv_get_phase_times", "dv_ccp_violation_noalloc",
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
                ("precision", C.c_int32), ("max_backtracks", C.c_int32), ("verbose", C.c_int32)]


class StepStats(C.Structure):
    _fields_ = [("num_contacts", C.c_int32), ("num_possible", C.c_int32),
                ("iterations", C.c_int32), ("backtracks", C.c_int32), ("residual", C.c_double),
                ("objective", C.c_double), ("elapsed_ms", C.c_double), ("time", C.c_double),
                ("time_index", C.c_int32), ("status", C.c_int32), ("collide_ms", C.c_double),
                ("solve_ms", C.c_double), ("sweeps", C.c_int32), ("pad_", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


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
        "dv_collide": [vp],
        "dv_get_state": [vp, dp, dp],
        "dv_set_state": [vp, dp, dp],
        "dv_get_contact_force": [vp, dp],
        "dv_get_num_contacts": [vp, ip, ip],
        "dv_get_contacts": [vp, up, up, dp, dp],
        "dv_get_gamma": [vp, dp, C.c_int32, ip],
        "dv_set_gamma": [vp, dp, C.c_int32],
        "dv_get_frames": [vp, dp],
        "dv_get_schur_vector": [vp, dp],
        "dv_ccp_violation": [vp, dp],
        "dv_energies": [vp, dp, dp],
        "dv_contact_forces_per_collision": [vp, dp, dp],
        "dv_get_step_stats": [vp, C.POINTER(StepStats)],
        "dv_get_step_history": [vp, C.POINTER(StepStats), C.c_int32, ip],
        "dv_clear_step_history": [vp],
        "dv_get_phase_times": [vp, dp, C.POINTER(C.c_int64), C.c_int32],
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
    o.max_backtracks = int(p.get("max_backtracks", o.max_backtracks))
    o.precision = int(p.get("precision", precision))
    o.verbose = int(p.get("verbose", 0))
    return o


def body_array(pos, vel, mass, geom, fixed, family):
    nb = int(np.asarray(pos).shape[0])
    arr = (BodyDesc * max(nb, 1))()
    pos = np.asarray(pos, dtype=np.float64)
    vel = np.asarray(vel, dtype=np.float64)
    geom = np.asarray(geom, dtype=np.float64)
    for i in range(nb):
        b = arr[i]
        b.pos[:] = pos[i].tolist()
        b.vel[:] = vel[i].tolist()
        b.mass = float(mass[i])
        b.geom[:] = geom[i].tolist()
        b.fixed = int(fixed[i])
        b.family = int(family[i])
    return arr, nb


class NativeScene:
    """One device-resident scene (dv_scene*) driven through the C ABI."""

    def __init__(self, pos, vel, mass, geom, fixed, family, params: dict,
                 precision=DV_PREC_FP64):
        L = lib()
        arr, nb = body_array(pos, vel, mass, geom, fixed, family)
        self.nb = nb
        self.params = make_params(params, precision)
        h = C.c_void_p()
        check(L.dv_scene_create(arr, nb, C.byref(self.params), C.byref(h)), "dv_scene_create")
        self.h = h

    @classmethod
    def from_scene(cls, scene, precision=DV_PREC_FP64, **overrides):
        p = dict(scene.params)
        p.update(overrides)
        return cls(scene.pos, scene.vel, scene.mass, scene.geom, scene.fixed, scene.family, p,
                   precision)

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
