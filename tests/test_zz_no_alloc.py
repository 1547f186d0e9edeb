"""dv_ccp_violation_noalloc: the CCP-violation diagnostic for callers that may
not allocate device memory (their memory belongs to their own pool, or their
loop cannot afford an allocation that may synchronise the device).  It reads
caller-owned device arrays and uses only a fixed scratch array compiled into
the library, so it must give exactly what the allocating dv_ccp_violation
gives for the same scene, call after call.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10  # the FP64 parity tolerance used by the other tests


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_violation_matches_allocating_entry_point(native):
    import torch

    L = native.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = torch.empty(4, dtype=torch.float64, device="cuda")
    for sc, steps in ((scenes.random_cluster(5, n=60), 4),
                      (scenes.settling_box(n_side=6, max_iterations=300), 150)):
        g = native.NativeScene.from_scene(sc)
        g.step(steps)
        want = g.ccp_violation()
        a, b, nP, _ = g.contacts()
        nc = a.size
        assert nc > 10
        gam = g.gamma()[:nc]
        _, v = g.state()
        d_gam = _dev(torch, gam, torch.float64)
        d_nP = _dev(torch, nP, torch.float64)
        d_a = _dev(torch, a.view(np.int32), torch.int32)
        d_b = _dev(torch, b.view(np.int32), torch.int32)
        d_v = _dev(torch, v, torch.float64)
        torch.cuda.synchronize()
        for _ in range(2):  # two calls in a row share the scratch array
            out.fill_(float("nan"))
            rc = L.dv_ccp_violation_noalloc(nc, sc.nb, _ptr(d_gam), _ptr(d_nP), _ptr(d_a),
                                            _ptr(d_b), _ptr(d_v), sc.params["mu"],
                                            sc.params["h"], _ptr(out), stream)
            assert rc == 0, native.lib().dv_last_error()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.abs(got - want) <= REL_TOL * np.maximum(np.abs(want), 1e-300))
            assert np.array_equal(got, want)
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
