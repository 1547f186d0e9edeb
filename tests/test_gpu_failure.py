"""Failure detection on the GPU without a fault: the solve kernels' bounded
waits (grid barrier, bulk-copy mbarrier) are run against conditions that never
come true and must end at their time limit with an error status the host
reads; the device stays usable."""
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
