"""dv_ccp_violation_noalloc: the CCP-violation diagnostic for callers that may
not allocate device memory (their memory belongs to their own pool, or their
loop cannot afford an allocation that may synchronise the device).  It reads
caller-owned device arrays and uses only a fixed scratch array compiled into
the library, so it must give exactly what the allocating dv_ccp_violation
gives for the same scene, call after call -- including the NaN and signed-zero
cases of its minima.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10  # the FP64 parity tolerance used by the other tests
TILE = 512       # contacts per reduction tile


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class _Call:
    """The device copies of one scene's contact arrays and the entry point."""

    def __init__(self, native, torch, g, sc):
        self.L = native.lib()
        self.torch = torch
        self.sc = sc
        a, b, nP, _ = g.contacts()
        self.nc = a.size
        _, v = g.state()
        self.d_nP = _dev(torch, nP, torch.float64)
        self.d_a = _dev(torch, a.view(np.int32), torch.int32)
        self.d_b = _dev(torch, b.view(np.int32), torch.int32)
        self.d_v = _dev(torch, v, torch.float64)
        self.out = torch.empty(4, dtype=torch.float64, device="cuda")
        self.stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def __call__(self, gamma, ida=None):
        d_gam = _dev(self.torch, gamma, self.torch.float64)
        d_a = self.d_a if ida is None else _dev(self.torch, ida.view(np.int32), self.torch.int32)
        self.torch.cuda.synchronize()
        self.out.fill_(12345.0)
        rc = self.L.dv_ccp_violation_noalloc(self.nc, self.sc.nb, _ptr(d_gam), _ptr(self.d_nP),
                                             _ptr(d_a), _ptr(self.d_b), _ptr(self.d_v),
                                             self.sc.params["mu"], self.sc.params["h"],
                                             _ptr(self.out), self.stream)
        assert rc == 0, self.L.dv_last_error()
        self.torch.cuda.synchronize()
        return self.out.cpu().numpy()


def _squeezed_box():
    """The 1,000-sphere settling box with its lattice squeezed so that ~1,800
    contacts (four reduction tiles) are active from the first step."""
    sc = scenes.settling_box(max_iterations=300)
    p = sc.pos.copy()
    p[5:, :2] *= 0.905
    p[5:, 2] = 0.05 + (p[5:, 2] - 0.06) * 0.905
    sc.pos = p
    return sc


def _check_equal(got, want):
    assert np.all((np.abs(got - want) <= REL_TOL * np.maximum(np.abs(want), 1e-300))
                  | (np.isnan(got) & np.isnan(want)))
    assert np.array_equal(got, want, equal_nan=True)
    assert np.array_equal(np.signbit(got), np.signbit(want))


def test_noalloc_violation_matches_allocating_entry_point(native):
    import torch

    # the second scene spans several reduction tiles (cross-tile folds)
    for sc, steps, min_nc in ((scenes.random_cluster(5, n=60), 4, 10),
                              (_squeezed_box(), 3, 2 * TILE)):
        g = native.NativeScene.from_scene(sc)
        g.step(steps)
        want = g.ccp_violation()
        call = _Call(native, torch, g, sc)
        assert call.nc > min_nc, call.nc
        gam = g.gamma()[:call.nc]
        for _ in range(2):  # two calls in a row share the scratch array
            _check_equal(call(gam), want)
        g.close()


def test_noalloc_violation_nan_and_signed_zero_like_allocating(native):
    """Planted impulses: the allocating path's minima come from a sequential
    host loop (a NaN first item is the result, later NaNs are passed over, the
    earlier of -0 and +0 is kept); the allocation-free one must agree."""
    import torch

    sc = _squeezed_box()
    g = native.NativeScene.from_scene(sc)
    g.step(3)
    call = _Call(native, torch, g, sc)
    nc = call.nc
    base = g.gamma()[:nc].copy()
    cases = []
    x = base.copy(); x[0, 0] = np.nan; cases.append(x)               # NaN first item
    x = base.copy(); x[nc // 2, 0] = np.nan; cases.append(x)         # NaN later
    x = base.copy(); x[:, 0] = np.abs(x[:, 0]) + 1.0; x[3, 0] = -0.0; x[nc - 7, 0] = 0.0
    cases.append(x)                                                  # -0 before +0
    x = base.copy(); x[:, 0] = np.abs(x[:, 0]) + 1.0; x[5, 0] = 0.0; x[TILE + 9, 0] = -0.0
    cases.append(x)                                                  # +0 before -0
    for gam in cases:
        g.set_gamma(gam)
        want = g.ccp_violation()
        _check_equal(call(gam), want)
    g.close()


def test_noalloc_violation_empty_and_bad_ids(native):
    import torch

    L = native.lib()
    sc = scenes.random_cluster(5, n=60)
    g = native.NativeScene.from_scene(sc)
    g.step(4)
    call = _Call(native, torch, g, sc)
    gam = g.gamma()[:call.nc]
    bad = g.contacts()[0].copy()
    bad[call.nc // 2] = sc.nb  # a body id past the last body: not read, result void
    got = call(gam, ida=bad)
    assert np.all(np.isnan(got)), got
    # no contacts: zeros, and the scratch array is not touched
    out = torch.full((4,), 7.0, dtype=torch.float64, device="cuda")
    rc = L.dv_ccp_violation_noalloc(0, sc.nb, None, None, None, None, None, 0.25, 1e-3,
                                    _ptr(out), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), np.zeros(4))
    g.close()


def test_noalloc_violation_rejects_oversize(native):
    import torch

    L = native.lib()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    ids = torch.zeros(4, dtype=torch.int32, device="cuda")
    too_many = 16777216 + 1
    rc = L.dv_ccp_violation_noalloc(too_many, 2, _ptr(buf), _ptr(buf), _ptr(ids), _ptr(ids),
                                    _ptr(buf), 0.25, 1e-3, _ptr(buf), None)
    assert rc == 1
    assert b"DV_NOALLOC_MAX_CONTACTS" in L.dv_last_error()
