"""ctypes front end of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of bench.py; the product package never imports it.
Parity unpinned: see dv_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "liboracle.so")

CUDA_INCLUDE = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
CFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
          "-fPIC", "-shared", "-std=c++17", "-Wall",
          # Thrust's OpenMP backend for the collision pass's bin sort (header-only)
          "-DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_OMP", "-I", CUDA_INCLUDE]


def build(force=False):
    """Compile oracle/dv_oracle.cpp into oracle/_ref/liboracle.so."""
    src = os.path.join(HERE, "dv_oracle.cpp")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(os.path.join(HERE, "dv_oracle.h"))):
        return LIB_PATH
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    subprocess.check_call(["g++", *CFLAGS, "-o", LIB_PATH, src])
    return LIB_PATH


class OrParams(C.Structure):
    _fields_ = [("h", C.c_double), ("mu", C.c_double), ("gravity", C.c_double * 3),
                ("envelope", C.c_double), ("tolerance", C.c_double),
                ("max_iterations", C.c_int), ("warm_start", C.c_int),
                ("reduce_mode", C.c_int), ("spmv_mode", C.c_int),
                ("max_backtracks", C.c_int), ("threads", C.c_int), ("apgd_mode", C.c_int),
                ("solver", C.c_int), ("anti_relaxation", C.c_int),
                ("fp64_narrowphase", C.c_int)]


class OrStats(C.Structure):
    _fields_ = [("num_contacts", C.c_int), ("num_possible", C.c_int), ("iterations", C.c_int),
                ("backtracks", C.c_int), ("residual", C.c_double), ("objective", C.c_double),
                ("status", C.c_int), ("gamma_size", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        up = C.POINTER(C.c_uint32)
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.c_int, dp, dp, dp, dp, ip, ip, C.POINTER(OrParams)]
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_set_params.argtypes = [C.c_void_p, C.POINTER(OrParams)]
        for name in ("or_step",):
            getattr(L, name).argtypes = [C.c_void_p, C.c_int]
        L.or_collide.argtypes = [C.c_void_p]
        L.or_solve.argtypes = [C.c_void_p]
        L.or_get_step_vectors.argtypes = [C.c_void_p, dp, dp, dp]
        L.or_get_stats.argtypes = [C.c_void_p, C.POINTER(OrStats)]
        L.or_get_state.argtypes = [C.c_void_p, dp, dp]
        L.or_set_state.argtypes = [C.c_void_p, dp, dp]
        L.or_get_fcontact.argtypes = [C.c_void_p, dp]
        L.or_get_gamma.argtypes = [C.c_void_p, dp, C.c_int]
        L.or_set_gamma.argtypes = [C.c_void_p, dp, C.c_int]
        L.or_get_contacts.argtypes = [C.c_void_p, up, up, dp, dp]
        L.or_get_frames.argtypes = [C.c_void_p, dp]
        L.or_get_r.argtypes = [C.c_void_p, dp]
        L.or_ccp_violation.argtypes = [C.c_void_p, dp]
        L.or_add_bilateral.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double]
        L.or_get_bilateral_gamma.argtypes = [C.c_void_p, dp]
        L.or_kinetic_energy.restype = C.c_double
        L.or_kinetic_energy.argtypes = [C.c_void_p]
        L.or_potential_energy.restype = C.c_double
        L.or_potential_energy.argtypes = [C.c_void_p]
        L.or_project.argtypes = [dp, C.c_double]
        L.or_frame.argtypes = [dp, dp, dp]
        L.or_length3.restype = C.c_double
        L.or_length3.argtypes = [dp]
        L.or_normalize3.argtypes = [dp, dp]
        L.or_ordered_sum.restype = C.c_double
        L.or_ordered_sum.argtypes = [dp, C.c_int64]
        L.or_schur.argtypes = [C.c_int, C.c_int, up, up, dp, dp, dp, dp, C.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _up(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def make_params(p: dict, reduce_mode=0, spmv_mode=0, threads=0, apgd_mode=0) -> OrParams:
    o = OrParams()
    o.h = p["h"]
    o.mu = p["mu"]
    o.gravity[:] = list(p["gravity"])
    o.envelope = p["envelope"]
    o.tolerance = p["tolerance"]
    o.max_iterations = int(p["max_iterations"])
    o.warm_start = int(p["warm_start"])
    o.reduce_mode = reduce_mode
    o.spmv_mode = spmv_mode
    o.max_backtracks = int(p.get("max_backtracks", 4096))
    o.threads = threads
    o.apgd_mode = apgd_mode
    o.solver = int(p.get("solver", 1))
    o.fp64_narrowphase = int(p.get("fp64_narrowphase", 0))
    o.anti_relaxation = int(p.get("anti_relaxation", 0))
    return o


class OracleScene:
    """One scene held by the CPU oracle; mirrors the state a System keeps."""

    def __init__(self, scene, reduce_mode=0, spmv_mode=0, threads=0, apgd_mode=0):
        L = lib()
        self.nb = scene.nb
        self._arrs = [np.ascontiguousarray(scene.pos, dtype=np.float64),
                      np.ascontiguousarray(scene.vel, dtype=np.float64),
                      np.ascontiguousarray(scene.mass, dtype=np.float64),
                      np.ascontiguousarray(scene.geom, dtype=np.float64),
                      np.ascontiguousarray(scene.fixed, dtype=np.int32),
                      np.ascontiguousarray(scene.family, dtype=np.int32)]
        a = self._arrs
        self.params = make_params(scene.params, reduce_mode, spmv_mode, threads, apgd_mode)
        self.h = L.or_create(self.nb, _dp(a[0]), _dp(a[1]), _dp(a[2]), _dp(a[3]), _ip(a[4]),
                             _ip(a[5]), C.byref(self.params))
        if getattr(scene, "gamma", None) is not None:
            self.set_gamma(scene.gamma)
        for row in getattr(scene, "bilateral", None) or ():
            self.add_bilateral(*row)

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    def step(self, n=1):
        return lib().or_step(self.h, n)

    def collide(self):
        return lib().or_collide(self.h)

    def solve(self):
        """Solver::solve() alone: no update, no clock."""
        return lib().or_solve(self.h)

    def stats(self):
        s = OrStats()
        lib().or_get_stats(self.h, C.byref(s))
        return {k: getattr(s, k) for k, _ in OrStats._fields_}

    def state(self):
        p = np.zeros((self.nb, 3))
        v = np.zeros((self.nb, 3))
        lib().or_get_state(self.h, _dp(p), _dp(v))
        return p, v

    def set_state(self, p, v):
        p = np.ascontiguousarray(p, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        lib().or_set_state(self.h, _dp(p), _dp(v))

    def fcontact(self):
        f = np.zeros((self.nb, 3))
        lib().or_get_fcontact(self.h, _dp(f))
        return f

    def gamma(self):
        n = lib().or_get_gamma(self.h, None, 0)
        g = np.zeros((max(n, 0), 3))
        if n:
            lib().or_get_gamma(self.h, _dp(g), n)
        return g

    def set_gamma(self, g):
        g = np.ascontiguousarray(g, dtype=np.float64).reshape(-1, 3)
        lib().or_set_gamma(self.h, _dp(g), g.shape[0])

    def contacts(self):
        nc = self.stats()["num_contacts"]
        a = np.zeros(nc, dtype=np.uint32)
        b = np.zeros(nc, dtype=np.uint32)
        nP = np.zeros((nc, 4))
        loc = np.zeros((nc, 3))
        if nc:
            lib().or_get_contacts(self.h, _up(a), _up(b), _dp(nP), _dp(loc))
        return a, b, nP, loc

    def frames(self):
        nc = self.stats()["num_contacts"]
        F = np.zeros((nc, 9))
        if nc:
            lib().or_get_frames(self.h, _dp(F))
        return F

    def r(self):
        nc = self.stats()["num_contacts"]
        r = np.zeros((nc, 3))
        if nc:
            lib().or_get_r(self.h, _dp(r))
        return r

    def add_bilateral(self, dof_a, dof_b=-1, velocity=0.0, start_time=0.0):
        """System::addBilateralConstraintDOF (before the first step)."""
        if lib().or_add_bilateral(self.h, int(dof_a), int(dof_b), float(velocity),
                                  float(start_time)) != 0:
            raise ValueError("bilateral DOF out of range")

    def bilateral_gamma(self):
        n = lib().or_get_bilateral_gamma(self.h, None)
        g = np.zeros(n)
        if n:
            lib().or_get_bilateral_gamma(self.h, _dp(g))
        return g

    def step_vectors(self):
        """r, b (bilateral rows first) and k (3 per body) of the last step."""
        n = 3 * self.stats()["num_contacts"] + len(self.bilateral_gamma())
        r, b, k = np.zeros(n), np.zeros(n), np.zeros(3 * self.nb)
        lib().or_get_step_vectors(self.h, _dp(r), _dp(b), _dp(k))
        return r, b, k

    def ccp_violation(self):
        o = np.zeros(4)
        lib().or_ccp_violation(self.h, _dp(o))
        return o

    def kinetic_energy(self):
        return lib().or_kinetic_energy(self.h)

    def potential_energy(self):
        return lib().or_potential_energy(self.h)


def project(x, mu):
    x = np.array(x, dtype=np.float64)
    lib().or_project(_dp(x), mu)
    return x


def frame(n):
    n = np.array(n, dtype=np.float64)
    u = np.zeros(3)
    v = np.zeros(3)
    lib().or_frame(_dp(n), _dp(u), _dp(v))
    return u, v


def length3(v):
    v = np.array(v, dtype=np.float64)
    return lib().or_length3(_dp(v))


def normalize3(v):
    v = np.array(v, dtype=np.float64)
    o = np.zeros(3)
    lib().or_normalize3(_dp(v), _dp(o))
    return o


def ordered_sum(v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    return lib().or_ordered_sum(_dp(v), v.size)


def schur(nb, a, b, F, minv, x, spmv_mode=0):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    F = np.ascontiguousarray(F, dtype=np.float64)
    minv = np.ascontiguousarray(minv, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    lib().or_schur(nb, a.size, _up(a), _up(b), _dp(F), _dp(minv), _dp(x), _dp(out), spmv_mode)
    return out
