"""Mixed precision (DV_PREC_MIXED) against the FP64 oracle.

The mixed path keeps frames, Jacobian and N gamma products, iterates and the
cone projection in FP32 and everything that needs FP64 (Schur vector, the
Lipschitz-test and residual sums, D^T gamma and the update) in FP64.  Stated
error, per teacher-forced step (both sides start every step from the oracle's
state and warm start), relative 2-norms:

  APGD tolerance 1e-6:  gamma <= 1e-4, v <= 5e-5   (measured ~2e-5 / ~3e-6)
  APGD tolerance 1e-4:  gamma <= 2e-3, v <= 1e-3   (measured ~4e-4 / ~1e-4)

At the looser tolerance the two solves stop at different iterates, so the
difference is the solver's own tolerance, not the precision.  The mixed
solve must also converge within the iteration cap whenever FP64 does
(tolerance 1e-4).  These scenes are statically indeterminate when they
settle (many impulse distributions give the same motion), so gamma is not
unique there.

On scenes where the FP64 solution is pinned -- two FP64 oracle solves of
the same step, one warm- and one cold-started, agree to better than 1e-5 at
tolerance 1e-8: a sliding ball (2e-7), a 5-sphere vertical stack in motion
(5.5e-6; a chain of n contacts on n spheres has unique impulses) and the
40-sphere cluster (3.7e-8) -- the bound is gamma <= 1e-5 and v <= 1e-5
relative to the FP64 oracle.  FP32 iterates alone stall near their rounding
floor at that tolerance (the cluster: ~4,400 FP32 iterations against ~640
FP64 ones, the cap reached), so the mixed solve runs FP64 refinement
iterations from the FP32 best iterate (dv_params.refine_iterations) once its
FP32 phase stops improving.  Longer chains are not pinned even in FP64
(warm against cold start at 1e-8: 10 spheres 1.1e-4, 20 spheres worse; the
smallest eigenvalue of N falls like 1/n^2), so they are not held to it."""
import numpy as np
import pytest

from dvide_b200 import scenes

pytestmark = pytest.mark.gpu

BOUNDS = {1e-6: (1e-4, 5e-5), 1e-4: (2e-3, 1e-3)}
DETERMINATE_TOL = 1e-8     # APGD tolerance at which the FP64 gamma is pinned
DETERMINATE_BOUND = 1e-5   # gamma and v, relative 2-norm against the FP64 oracle
REFINE_ITERATIONS = 2000


def _rel(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n > 0 else float(np.linalg.norm(a - b))


@pytest.mark.parametrize("tol", [1e-4, 1e-6])
@pytest.mark.parametrize("which", ["cluster", "box"])
def test_mixed_error_against_fp64_oracle(native, oracle_mod, tol, which):
    if which == "cluster":
        sc, steps = scenes.random_cluster(0, n=40, max_iterations=2000), 8
    else:
        sc, steps = scenes.settling_box(n_side=6, max_iterations=1000), 60
    g = native.NativeScene.from_scene(sc, precision=1, tolerance=tol)
    o = oracle_mod.OracleScene(sc)
    o.params = oracle_mod.make_params({**sc.params, "tolerance": tol})
    oracle_mod.lib().or_set_params(o.h, o.params)
    gmax, vmax, solved = 0.0, 0.0, 0
    for k in range(steps):
        p, v = o.state()
        g.set_state(p, v)
        g.set_gamma(o.gamma())
        o.step(1)
        g.step(1)
        so, sg = o.stats(), g.stats()
        assert sg["num_contacts"] == so["num_contacts"], k
        if so["num_contacts"] == 0:
            continue
        solved += 1
        gmax = max(gmax, _rel(g.gamma(), o.gamma()))
        vmax = max(vmax, _rel(g.state()[1], o.state()[1]))
        if tol == 1e-4 and so["iterations"] < sc.params["max_iterations"]:
            assert sg["iterations"] < sc.params["max_iterations"], (k, so, sg)
    assert solved > 0
    gb, vb = BOUNDS[tol]
    assert gmax <= gb and vmax <= vb, (gmax, vmax)


def test_mixed_batch_equals_mixed_alone(native):
    rng = np.random.default_rng(2)
    scs = [scenes.random_cluster(1, n=30), scenes.lattice_container(rng, 150),
           scenes.settling_box(n_side=3)]
    b = native.NativeBatch(scs, precision=1)
    b.step(10)
    for i, sc in enumerate(scs):
        g = native.NativeScene.from_scene(sc, precision=1)
        g.step(10)
        assert np.array_equal(b.state(i)[0], g.state()[0]), i
        assert np.array_equal(b.gamma(i), g.gamma()), i


def _determinate(which):
    """Scenes whose FP64 impulses are pinned at tolerance 1e-8, in motion (so
    that relative velocity errors are measured against a velocity that is not
    noise)."""
    if which == "ball":
        # sliding on the ground (friction on the cone surface), slowly enough
        # that the cone's normal lift mu |v_t| stays below g h: it keeps contact
        sc = scenes.ball_on_ground(h=1e-2, tolerance=DETERMINATE_TOL, warm_start=1)
        sc.vel[1] = (0.2, 0.0, 0.1)
        return sc, 5
    if which == "stack5":
        sc = scenes.sphere_stack(5, tolerance=DETERMINATE_TOL)
        sc.vel[1:] = (0.1, 0.0, -0.05)   # the stack drops and slides on the floor
        return sc, 20
    return scenes.random_cluster(0, n=40, max_iterations=5000, tolerance=DETERMINATE_TOL), 8


@pytest.mark.parametrize("which", ["ball", "stack5", "cluster40"])
def test_mixed_refined_within_1e5_on_determinate_scenes(native, oracle_mod, which):
    sc, steps = _determinate(which)
    g = native.NativeScene.from_scene(sc, precision=1, refine_iterations=REFINE_ITERATIONS)
    o = oracle_mod.OracleScene(sc)
    gmax, vmax, solved, refined = 0.0, 0.0, 0, 0
    for k in range(steps):
        p, v = o.state()
        g.set_state(p, v)
        g.set_gamma(o.gamma())
        o.step(1)
        g.step(1)
        so, sg = o.stats(), g.stats()
        assert sg["num_contacts"] == so["num_contacts"], k
        if so["num_contacts"] == 0:
            continue
        solved += 1
        refined += sg["refine_iterations"] > 0
        if so["residual"] < DETERMINATE_TOL:  # FP64 converged: so must the mixed solve
            assert sg["residual"] < DETERMINATE_TOL, (k, sg)
        vo = o.state()[1]
        assert np.linalg.norm(vo) > 1e-2  # a velocity of the scene, not rounding noise
        gmax = max(gmax, _rel(g.gamma(), o.gamma()))
        vmax = max(vmax, _rel(g.state()[1], vo))
    assert solved > 0
    assert gmax <= DETERMINATE_BOUND and vmax <= DETERMINATE_BOUND, (gmax, vmax, refined)


def test_refinement_off_is_the_plain_mixed_solve(native):
    """refine_iterations = 0 (the default) launches the FP32 kernel alone: the
    same bits as before the option existed, i.e. as a second scene without it;
    with refinement on, a solve that converges in FP32 is not touched."""
    sc = scenes.random_cluster(3, n=40, tolerance=1e-4)
    a = native.NativeScene.from_scene(sc, precision=1)
    b = native.NativeScene.from_scene(sc, precision=1, refine_iterations=0)
    c = native.NativeScene.from_scene(sc, precision=1, refine_iterations=100)
    for _ in range(6):
        a.step(1)
        b.step(1)
        c.step(1)
        assert np.array_equal(a.state()[1], b.state()[1])
        sa, sc_ = a.stats(), c.stats()
        if sa["num_contacts"] and sa["residual"] < 1e-4:
            assert sc_["refine_iterations"] == 0
            assert np.array_equal(a.gamma(), c.gamma())
            assert np.array_equal(a.state()[1], c.state()[1])


def test_refined_batch_equals_refined_alone(native):
    """FP64 refinement in a batch: each scene's result is the same bits as the
    scene stepped alone with refinement (the refinement launch, like the FP32
    one, works per scene), including scenes whose FP32 phase converges and
    scenes that need FP64 iterations."""
    rng = np.random.default_rng(4)
    scs = [scenes.random_cluster(1, n=30, tolerance=1e-8, max_iterations=3000),
           scenes.lattice_container(rng, 150, tolerance=1e-6),
           scenes.settling_box(n_side=3)]
    b = native.NativeBatch(scs, precision=1, refine_iterations=REFINE_ITERATIONS)
    b.step(10)
    hist, _ = b.history()
    refined = 0
    for i, sc in enumerate(scs):
        g = native.NativeScene.from_scene(sc, precision=1, refine_iterations=REFINE_ITERATIONS)
        for k in range(10):
            g.step(1)
            st = g.stats()
            refined += st["refine_iterations"] > 0
            # the batch's per-scene report of the same step (dv_batch_step_history)
            assert hist[k][i]["refine_iterations"] == st["refine_iterations"], (i, k)
            assert hist[k][i]["iterations"] == st["iterations"], (i, k)
        assert np.array_equal(b.state(i)[0], g.state()[0]), i
        assert np.array_equal(b.state(i)[1], g.state()[1]), i
        assert np.array_equal(b.gamma(i), g.gamma()), i
    assert refined > 0


def test_refinement_with_scenes_without_contacts(native):
    """A refined batch holding a scene without contacts (free flight) and
    scenes whose FP32 phase converges: each steps as it does alone."""
    scs = [scenes.free_balls(n=3, tolerance=1e-6),
           scenes.random_cluster(2, n=27, tolerance=1e-4),
           scenes.ball_on_ground(h=1e-3, tolerance=1e-8, warm_start=1)]
    b = native.NativeBatch(scs, precision=1, refine_iterations=REFINE_ITERATIONS)
    b.step(6)
    for i, sc in enumerate(scs):
        g = native.NativeScene.from_scene(sc, precision=1, refine_iterations=REFINE_ITERATIONS)
        g.step(6)
        assert np.array_equal(b.state(i)[0], g.state()[0]), i
        assert np.array_equal(b.state(i)[1], g.state()[1]), i
    assert b.scene_stats()[0]["num_contacts"] == 0
