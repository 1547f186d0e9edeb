"""Physics sanity checks the reference's drivers print (they have no automated
tests): at rest the contact forces carry the weight.  models/test_oneBall.cu
checks the ground's normal force on a resting ball against m g, and
models/test_compaction.cu:403-408 sums the container's vertical contact force
against the weight of what it holds.  Here both run on the GPU path, with the
FP64 solve and with mixed precision plus FP64 refinement; f_contact is
D^T gamma / h for every body, fixed ones included (System.cu:570-573), so
the forces on all bodies also sum to zero."""
import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu

G = 9.81


@pytest.mark.parametrize("precision,refine", [(0, 0), (1, 500)], ids=["fp64", "mixed_refined"])
def test_ball_on_ground_carries_its_weight(native, precision, refine):
    sc = scenes.ball_on_ground(h=1e-3)  # gravity along -y; body 0 is the ground
    g = native.NativeScene.from_scene(sc, precision=precision, refine_iterations=refine)
    g.step(200)
    f = g.fcontact()
    mg = sc.mass[1] * G
    assert abs(f[1, 1] - mg) <= 1e-4 * mg and abs(f[0, 1] + mg) <= 1e-4 * mg
    assert np.abs(f.sum(axis=0)).max() <= 1e-9 * mg
    g.close()


@pytest.mark.parametrize("precision,refine,tol", [(0, 0, 5e-3), (1, 500, 1e-2)],
                         ids=["fp64", "mixed_refined"])
def test_settled_box_walls_carry_the_weight(native, precision, refine, tol):
    """The 1,000-sphere settling box (C0 settings) at rest from step 300 on:
    every 100 steps the floor and walls carry the spheres' weight within tol,
    and within tol / 2 on average (the oracle, to which the FP64 path is
    bit-identical, gives 0.9996, 0.9977, 1.0012, 1.0018, 0.9971, 1.0007 at
    steps 300 to 800)."""
    sc = scenes.settling_box()
    g = native.NativeScene.from_scene(sc, precision=precision, refine_iterations=refine)
    g.step(300)
    fixed = sc.fixed == 1
    weight = sc.mass[~fixed].sum() * G
    ratios = []
    for _ in range(5):
        g.step(100)
        f = g.fcontact()
        ratios.append(-f[fixed, 2].sum() / weight)
        assert abs(f[:, 2].sum()) <= 1e-9 * weight
        _, v = g.state()
        assert np.abs(v).max() < 2e-3  # at rest
    assert all(abs(r - 1.0) < tol for r in ratios), ratios
    assert abs(np.mean(ratios) - 1.0) < tol / 2, ratios
    g.close()
