"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bar: bit-exact for the contact list (ids, normal, gap, location, frame) and,
because both sides share one floating-point order, bit-exact for the FP64
solve too (gamma, v, p, contact forces, iteration count, residual); the
parity tolerance (1e-10 relative on gamma and v) is asserted as well so a
failure reports its size."""
import numpy as np
import pytest

from dvide_b200 import scenes, workloads

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10  # plain FP64 parity bar on gamma and body velocities


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm(a - b)
    n = np.linalg.norm(b)
    return d / n if n > 0 else d


def _pair(native, oracle_mod, sc, **kw):
    g = native.NativeScene.from_scene(sc, **kw)
    o = oracle_mod.OracleScene(sc)
    if kw:
        o.params = oracle_mod.make_params({**sc.params, **kw})
        oracle_mod.lib().or_set_params(o.h, o.params)
    return g, o


def _compare_contacts(g, o):
    ga, gb, gnP, gloc = g.contacts()
    oa, ob, onP, oloc = o.contacts()
    assert np.array_equal(ga, oa) and np.array_equal(gb, ob)
    assert np.array_equal(gnP, onP)
    assert np.array_equal(gloc, oloc)
    return ga.size


@pytest.mark.parametrize("seed", [0, 1, 2, 3, 4])
def test_collide_bitexact(native, oracle_mod, seed):
    sc = scenes.random_cluster(seed, n=60)
    g, o = _pair(native, oracle_mod, sc)
    g.collide()
    o.collide()
    nc = _compare_contacts(g, o)
    assert nc > 20
    assert np.array_equal(g.frames(), o.frames())
    assert g.num_contacts()[1] == o.stats()["num_possible"]


def test_collide_settling_box_bitexact(native, oracle_mod):
    sc = scenes.settling_box()
    g, o = _pair(native, oracle_mod, sc)
    # squeeze the lattice so that many neighbours are in contact
    p = sc.pos.copy()
    p[5:, :2] *= 0.905
    p[5:, 2] = 0.05 + (p[5:, 2] - 0.06) * 0.905
    g.set_state(p, sc.vel)
    o.set_state(p, sc.vel)
    g.collide()
    o.collide()
    nc = _compare_contacts(g, o)
    assert nc > 1000


def _teacher_forced(native, oracle_mod, sc, steps, check_every=1, **kw):
    g, o = _pair(native, oracle_mod, sc, **kw)
    worst = 0.0
    solved = 0
    for k in range(steps):
        p, v = o.state()
        g.set_state(p, v)
        g.set_gamma(o.gamma())
        o.step(1)
        g.step(1)
        so, sg = o.stats(), g.stats()
        assert sg["num_contacts"] == so["num_contacts"], k
        if k % check_every:
            continue
        pg, vg = g.state()
        po, vo = o.state()
        gg, go = g.gamma(), o.gamma()
        assert _rel(gg, go) <= REL_TOL and _rel(vg, vo) <= REL_TOL, k
        assert np.array_equal(gg, go), (k, _rel(gg, go))
        assert np.array_equal(vg, vo), k
        assert np.array_equal(pg, po), k
        assert np.array_equal(g.fcontact(), o.fcontact()), k
        if so["num_contacts"]:
            solved += 1
            assert sg["iterations"] == so["iterations"], k
            assert sg["residual"] == so["residual"], k
            assert sg["objective"] == so["objective"], k
            assert sg["backtracks"] == so["backtracks"], k
        worst = max(worst, _rel(gg, go))
    return solved


def test_ball_on_ground_bitexact(native, oracle_mod):
    sc = scenes.ball_on_ground()
    assert _teacher_forced(native, oracle_mod, sc, 5) == 5


@pytest.mark.parametrize("seed", [0, 3])
def test_cluster_teacher_forced(native, oracle_mod, seed):
    sc = scenes.random_cluster(seed, n=40)
    assert _teacher_forced(native, oracle_mod, sc, 12) >= 10


def test_cluster_no_warm_start_and_frictionless(native, oracle_mod):
    sc = scenes.random_cluster(11, n=30, warm_start=0)
    assert _teacher_forced(native, oracle_mod, sc, 4) >= 3
    sc = scenes.random_cluster(12, n=30, mu=0.0)
    assert _teacher_forced(native, oracle_mod, sc, 4) >= 3


def test_settling_box_free_running_identical(native, oracle_mod):
    """A 216-sphere settling box run free for 150 steps stays bit-identical."""
    sc = scenes.settling_box(n_side=6, max_iterations=300)
    g, o = _pair(native, oracle_mod, sc)
    for k in range(150):
        o.step(1)
        g.step(1)
        assert g.stats()["num_contacts"] == o.stats()["num_contacts"], k
    pg, vg = g.state()
    po, vo = o.state()
    assert np.array_equal(pg, po) and np.array_equal(vg, vo)
    assert np.array_equal(g.gamma(), o.gamma())
    assert np.array_equal(g.ccp_violation(), o.ccp_violation())
    ke, pe = g.energies()
    assert ke == o.kinetic_energy() and pe == o.potential_energy()
    hist = g.history()
    assert len(hist) == 150


def test_c0_settling_teacher_forced(native, oracle_mod):
    """The 1,000-sphere settling box: bit-exact per step once the pile is in
    contact (states taken from the oracle's own trajectory)."""
    sc = scenes.settling_box()
    o = oracle_mod.OracleScene(sc)
    o.step(60)   # spheres reach the floor / each other
    p, v = o.state()
    sc2 = sc.copy()
    sc2.pos, sc2.vel = p, v
    g, o2 = _pair(native, oracle_mod, sc2)
    o2.set_gamma(o.gamma())
    assert _teacher_forced_from(native, g, o2, 8) >= 6


def _teacher_forced_from(native, g, o, steps):
    solved = 0
    for k in range(steps):
        p, v = o.state()
        g.set_state(p, v)
        g.set_gamma(o.gamma())
        o.step(1)
        g.step(1)
        so, sg = o.stats(), g.stats()
        assert sg["num_contacts"] == so["num_contacts"]
        assert np.array_equal(g.gamma(), o.gamma()), k
        pg, vg = g.state()
        po, vo = o.state()
        assert np.array_equal(vg, vo) and np.array_equal(pg, po), k
        if so["num_contacts"]:
            solved += 1
            assert sg["iterations"] == so["iterations"]
    return solved


def test_positional_warm_start(native, oracle_mod):
    """gamma_d is resized positionally: the prefix survives, growth is zero
    (APGD.cu:166); a step without contacts leaves it untouched."""
    sc = scenes.random_cluster(21, n=30)
    g, o = _pair(native, oracle_mod, sc)
    g.step(2)
    o.step(2)
    n0 = g.gamma().shape[0]
    # shrink the buffer, then grow back through the next solve
    short = o.gamma()[: max(1, n0 // 3)] * 0.5
    g.set_gamma(short)
    o.set_gamma(short)
    g.step(1)
    o.step(1)
    assert np.array_equal(g.gamma(), o.gamma())
    # lift every sphere out of contact: no solve, gamma unchanged
    p, v = o.state()
    p2 = p.copy()
    dyn = np.nonzero(sc.fixed == 0)[0]
    p2[dyn] = np.stack([np.arange(dyn.size) * 1.0, np.zeros(dyn.size), np.full(dyn.size, 5.0)], 1)
    before = o.gamma()
    g.set_state(p2, v)
    o.set_state(p2, v)
    g.step(1)
    o.step(1)
    assert g.stats()["num_contacts"] == 0
    assert np.array_equal(g.gamma(), before) and np.array_equal(o.gamma(), before)


def test_contact_force_outputs(native, oracle_mod):
    sc = scenes.random_cluster(8, n=30)
    g, o = _pair(native, oracle_mod, sc)
    g.step(3)
    o.step(3)
    n, f = g.contact_forces()
    F = o.frames()
    gam = o.gamma()
    h = sc.params["h"]
    assert np.array_equal(n, (gam[:, :1] * F[:, 0:3]) / h)
    assert np.allclose(f, (gam[:, 1:2] * F[:, 3:6] + gam[:, 2:3] * F[:, 6:9]) / h, rtol=0,
                       atol=1e-12)
    assert np.array_equal(g.r(), o.r())


def test_repeatable_bits(native):
    """Two runs of the same scene give identical bits (no atomics in any
    floating-point reduction)."""
    sc = scenes.settling_box(n_side=5, max_iterations=200)
    out = []
    for _ in range(2):
        g = native.NativeScene.from_scene(sc)
        g.step(80)
        out.append(g.state() + (g.gamma(),))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def _free_running(native, oracle_mod, sc, steps):
    """Both sides step the same scene on their own; every step bit-identical."""
    g, o = _pair(native, oracle_mod, sc)
    for k in range(steps):
        assert o.step(1) == 0, k
        g.step(1)
        so, sg = o.stats(), g.stats()
        assert sg["num_contacts"] == so["num_contacts"], k
        for key in ("iterations", "backtracks", "residual", "objective"):
            assert sg[key] == so[key], (k, key)
        assert np.array_equal(g.gamma(), o.gamma()), k
        pg, vg = g.state()
        po, vo = o.state()
        assert np.array_equal(vg, vo) and np.array_equal(pg, po), k
        assert np.array_equal(g.ccp_violation(), o.ccp_violation()), k
    return o.stats()


@pytest.mark.parametrize("n_around", [9, 16, 17, 40, 128, 129, 200, 400, 500])
def test_crowd_many_contacts_per_body_free_running(native, oracle_mod, n_around):
    """One free sphere overlapped by n_around others, which overlap many of
    each other too: body gathers walk from a few to hundreds of incidence
    entries (sixteen per load group, q in two halves of eight, ragged ends),
    and from 129 on, spheres with more than 128 partners with larger ids
    have their contacts written by k_sphere_pairs_wide (1, 59, 248 and 359
    such spheres for 129, 200, 400 and 500; its 256 CTAs take them in turn).
    Bit-identical to the oracle over three steps while the crowd flies apart:
    the first step's solve runs its 50 iterations, and by the third step few
    pairs are still in contact."""
    sc = scenes.crowd(n_around)
    g, o = _pair(native, oracle_mod, sc)
    g.collide()
    o.collide()
    _compare_contacts(g, o)
    ga = g.contacts()[0]
    assert np.count_nonzero(ga == 0) == n_around
    g.close()
    st = _free_running(native, oracle_mod, sc, 3)
    assert st["num_contacts"] < ga.size // 100 + 1


@pytest.mark.parametrize("n,ballast", [(8192, 8200), (8193, 0)], ids=["gridded", "large"])
def test_raspberry_many_partners_free_running(native, oracle_mod, n, ballast):
    """One sphere with n small ones on its surface.  Gridded (the ballast
    raises the median radius), its 8,192 partners are the most the wide pair
    kernel keeps for one sphere: a full 8,192-entry bitonic sort.  Without
    ballast it is above four times the median radius and is paired against
    every body of the scene, with no partner limit.  Either way the contact
    list and the first step (a 5-iteration solve) are bit-identical to the
    oracle.  (On the next step every contact separates; with 8,193 spheres on
    the every-body path the reference's APGD then ends that solve on a
    non-finite objective, in the oracle as on the GPU.)"""
    sc = scenes.raspberry(n, ballast=ballast)
    g, o = _pair(native, oracle_mod, sc)
    g.collide()
    o.collide()
    assert _compare_contacts(g, o) == n
    g.close()
    st = _free_running(native, oracle_mod, sc, 1)
    assert st["num_contacts"] == n and st["iterations"] > 0


def test_driver_moved_wall_free_running(native, oracle_mod):
    """A fixed wall moved between steps by the driver, as the reference's shear
    driver moves its boxes (models/test_shear.cu:389-406: the fixed boxes' v
    overwritten, p advanced by h v before DoTimeStep).  The wall's new position
    enters the next collision pass.  Its overwritten v enters neither k nor r:
    k = M v with M = 0 for a fixed body (System.cu:1411-1417, 1505).  The update
    sets it back to 0 (v = Minv (k + D^T gamma), :572, 577), so the step's
    p += h v (:581) leaves the wall where the driver put it.  Bit-identical to the oracle over 60 steps:
    the wall starts 1 mm from the lattice and pushes into it at 0.2 m/s while
    the lattice lands on the floor."""
    sc = scenes.settling_box()
    wall = 1  # open_box order: floor, -x wall, +x wall, -y wall, +y wall
    assert sc.fixed[wall] == 1
    sph = sc.fixed == 0
    p = sc.pos.copy()
    p[wall, 0] = (p[sph, 0] - sc.geom[sph, 0]).min() - 1e-3 - sc.geom[wall, 0]
    sc.pos = p
    g, o = _pair(native, oracle_mod, sc)
    h = sc.params["h"]
    on_wall = 0
    for k in range(60):
        p, v = o.state()
        v[wall] = (0.2, 0.0, 0.0)
        p[wall] = p[wall] + h * v[wall]
        o.set_state(p, v)
        g.set_state(p, v)
        assert o.step(1) == 0, k
        g.step(1)
        so, sg = o.stats(), g.stats()
        assert sg["num_contacts"] == so["num_contacts"], k
        for key in ("iterations", "backtracks", "residual", "objective"):
            assert sg[key] == so[key], (k, key)
        assert np.array_equal(g.gamma(), o.gamma()), k
        pg, vg = g.state()
        po, vo = o.state()
        assert np.array_equal(vg, vo) and np.array_equal(pg, po), k
        assert np.array_equal(g.fcontact(), o.fcontact()), k
        assert (vo[wall] == 0.0).all() and np.array_equal(po[wall], p[wall]), k
        ga, gb = g.contacts()[:2]
        on_wall = max(on_wall, int(np.count_nonzero((ga == wall) | (gb == wall))))
    assert on_wall > 20 and so["num_contacts"] > 100


def test_c0_compressed_free_running(native, oracle_mod):
    """The 1,000-sphere settling box (C0 settings: mu 0.25, h 1e-3, tolerance 1e-4,
    1,000 iterations, warm start) with the lattice squeezed so that ~1,800 contacts
    are active from the first step, free running for 25 steps while it springs apart."""
    sc = scenes.settling_box()
    p = sc.pos.copy()
    p[5:, :2] *= 0.905
    p[5:, 2] = 0.05 + (p[5:, 2] - 0.06) * 0.905
    sc.pos = p
    st = _free_running(native, oracle_mod, sc, 25)
    assert st["num_contacts"] > 100


def test_column_sample_free_running(native, oracle_mod):
    """The lowest 5,000 spheres of the settled 200,000-sphere column (its
    settings: mu 0.3, h 5e-4, tolerance 1e-4, 500 iterations, warm start):
    ~16,400 contacts, free running for 6 steps."""
    d = np.load(workloads.COLUMN_FILE)
    order = np.argsort(d["pos"][:, 2])[:5000]
    sc = workloads._column_scene(d["pos"][order].astype(np.float64),
                                 d["radius"][order].astype(np.float64), float(d["wall_height"]))
    st = _free_running(native, oracle_mod, sc, 6)
    assert st["num_contacts"] > 15000


def test_column_full_scale_contacts_and_one_step(native, oracle_mod):
    """The whole settled 200,000-sphere column that the benchmark times
    (~741,000 contacts): collision detection's contact list (ids, normal and
    gap, location) and tangent frames bit-identical to the oracle's
    (CollisionDetector.cu:547-665), then one full step from the same state and
    warm start (the 500-iteration APGD solve and the update, System.cu:544-583):
    gamma, v, p, iterations, backtracks and residual identical."""
    sc = workloads.column_settled()
    g, o = _pair(native, oracle_mod, sc)
    g.collide()
    o.collide()
    nc = _compare_contacts(g, o)
    assert nc > 700000
    assert np.array_equal(g.frames(), o.frames())
    assert g.num_contacts()[1] == o.stats()["num_possible"]
    g.step(1)
    o.step(1)
    so, sg = o.stats(), g.stats()
    assert sg["num_contacts"] == so["num_contacts"]
    for key in ("iterations", "backtracks", "residual", "objective"):
        assert sg[key] == so[key], key
    gg, go = g.gamma(), o.gamma()
    pg, vg = g.state()
    po, vo = o.state()
    assert _rel(gg, go) <= REL_TOL and _rel(vg, vo) <= REL_TOL
    assert np.array_equal(gg, go)
    assert np.array_equal(vg, vo) and np.array_equal(pg, po)


def test_diagnostics_after_the_step_records_grow(native, oracle_mod):
    """The CCP violation and energies read back through a pinned buffer that
    must survive the growth of the per-step record ring (a long dv_step call
    after a short one)."""
    sc = scenes.random_cluster(9, n=30)
    g, o = _pair(native, oracle_mod, sc)
    g.step(1)
    o.step(1)
    assert np.array_equal(g.ccp_violation(), o.ccp_violation())
    g.step(40)
    o.step(40)
    assert np.array_equal(g.ccp_violation(), o.ccp_violation())
    ke, pe = g.energies()
    assert ke == o.kinetic_energy() and pe == o.potential_energy()
