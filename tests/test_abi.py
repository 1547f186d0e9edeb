"""The C-ABI library loads and exports every entry point of include/dvide.h;
argument validation works without a GPU."""
import ctypes as C
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "dvide.h")).read()
    return sorted(set(re.findall(r"DV_API\s+[\w\s\*]+?\b(dv_\w+)\s*\(", src)))


def test_exports_match_header(native):
    L = native.lib()
    names = _declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert sorted(native.EXPORTS) == names


def test_defaults_are_reference_defaults(native):
    p = native.Params()
    assert native.lib().dv_params_default(C.byref(p)) == 0
    assert p.h == 1e-3 and p.mu == 0.25 and list(p.gravity) == [0.0, -9.81, 0.0]
    assert p.envelope == 1e-3 and p.tolerance == 1e-4 and p.max_iterations == 100000
    assert p.warm_start == 0 and p.solver == 1


def test_invalid_arguments_rejected_before_device_use(native):
    L = native.lib()
    arr, nb, _rec = native.body_array(np.zeros((1, 3)), np.zeros((1, 3)), [1.0], [[0.1, 0, 0]], [0],
                                      [-1])
    out = C.c_void_p()
    p = native.Params()
    L.dv_params_default(C.byref(p))
    p.h = -1.0
    assert L.dv_scene_create(arr, nb, C.byref(p), C.byref(out)) == 1
    L.dv_params_default(C.byref(p))
    p.solver = 3
    assert L.dv_scene_create(arr, nb, C.byref(p), C.byref(out)) == 7
    L.dv_params_default(C.byref(p))
    arr[0].mass = 0.0
    assert L.dv_scene_create(arr, nb, C.byref(p), C.byref(out)) == 1
    assert L.dv_step(None, 1) == 1
    assert L.dv_status_string(3) == b"non-finite value in the solve"


def test_missing_library_fails_loudly(monkeypatch, native):
    monkeypatch.setattr(native, "_lib", None)
    monkeypatch.setattr(native, "LIB_PATH", "/nonexistent/libdvide_b200.so")
    try:
        native.lib()
    except RuntimeError as e:
        assert "not built" in str(e)
    else:
        raise AssertionError("expected a RuntimeError")
