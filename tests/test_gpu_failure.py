"""Failure detection on the GPU without a fault: the solve kernels' bounded
waits (grid barrier, bulk-copy mbarrier) are run against conditions that never
come true and must end at their time limit with an error status the host
reads; the device stays usable."""
import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu


def test_bounded_waits_end_and_report(native):
    barrier, copy, bits = native.selftest_bounded_waits(50)
    assert barrier == 1 and copy == 1
    assert bits & 1 and bits & 32   # barrier timeout, copy timeout
    # the context is still usable: a normal step right after
    g = native.NativeScene.from_scene(scenes.ball_on_ground())
    g.step(3)
    assert g.stats()["num_contacts"] == 1 and g.stats()["status"] == 0
    g.close()


def test_selftest_rejects_bad_limit(native):
    with pytest.raises(Exception):
        native.selftest_bounded_waits(0)


def test_partner_limit_reports_an_argument_error(native):
    """A gridded sphere with more than 128 partners with larger ids is
    written by the wide pair kernel, which keeps at most 8,192 partners of one
    sphere.  A sphere with 8,192 small ones on its surface steps; with 8,193
    the step is reported as DV_ERR_ARG with a message, does nothing, and the
    scene stays usable.  (The ballast makes the big sphere a gridded one; see
    scenes.raspberry.)"""
    ok = native.NativeScene.from_scene(scenes.raspberry(8192, ballast=8200))
    ok.step(1)
    assert ok.stats()["num_contacts"] == 8192 and ok.stats()["status"] == 0
    bad = native.NativeScene.from_scene(scenes.raspberry(8193, ballast=8200))
    p0, v0 = bad.state()
    with pytest.raises(native.DvError) as e:
        bad.step(1)
    assert e.value.status == 1 and "8192 contact partners" in str(e.value)
    p1, v1 = bad.state()
    assert (p0 == p1).all() and (v0 == v1).all()
    # usable: the small spheres moved away, it steps
    p2 = p0.copy()
    p2[1:] *= 1.5
    bad.set_state(p2, v0)
    bad.step(1)
    assert bad.stats()["status"] == 0 and bad.stats()["num_contacts"] == 0
    ok.close()
    bad.close()
