"""Seeded synthetic scenes for the rigid-body contact step.

Every scene is a set of bodies in the layout DVIDE's ``System::initializeSystem``
flattens (src/System.cu:342-424): position, velocity, mass, contact geometry
``(r, 0, 0)`` for a sphere or box half-extents ``(hx, hy, hz)`` (src/Body.cuh:18-60),
a fixed flag and a collision family (src/PhysicsItem.cuh:13-33).

Workloads (no dataset exists for this path; all inputs are generated here):

* :func:`settling_box` -- 1,000 spheres r = 0.05 m, rho = 2600, on a 10x10x10
  lattice of spacing 0.11 m with +-0.005 m jitter, in an open box of 5 fixed
  boxes (floor 1.2 x 1.2 m interior, walls 1.5 m high), mu = 0.25, h = 1e-3.
  The reference analogue is models/test_compaction.cu:272-333 (boxes first,
  then spheres), with the sphere mass set to rho * 4/3 pi r^3 as in
  models/test_shear.cu:329.
* :func:`poured_column` -- 200,000 spheres, r ~ U[0.004, 0.006] m, rho = 2500,
  mu = 0.3, random sequential addition (rejection sampling) in a column of
  0.4 x 0.4 m cross-section, h = 5e-4.  The column is taller than 1.0 m because
  200,000 such spheres occupy 0.109 m^3, which no non-overlapping random
  packing fits into 0.16 m^3; the settled pile is about 1.1 m high.
* :func:`batch_scenes` -- independent settling scenes with log-uniform sphere
  counts, r ~ U[0.004, 0.006], mu ~ U[0.1, 0.5], each in its own container.
* :func:`ball_on_ground` -- models/test_oneBall.cu:240-283 (unit ball resting
  on a fixed box; at rest the normal impulse is m g h).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

G = 9.81


@dataclasses.dataclass
class Scene:
    pos: np.ndarray
    vel: np.ndarray
    mass: np.ndarray
    geom: np.ndarray
    fixed: np.ndarray
    family: np.ndarray
    params: dict
    name: str = "scene"
    # impulses of the previous solve (nc x 3, in that solve's contact order),
    # the warm start the first step reads: System::gamma_d carried over
    gamma: np.ndarray | None = None
    # bilateral DOF rows (System::addBilateralConstraintDOF): tuples
    # (dof_a, dof_b, velocity, start_time), DOF 3 i + k = axis k of body i
    bilateral: list | None = None

    @property
    def nb(self) -> int:
        return int(self.pos.shape[0])

    def copy(self) -> "Scene":
        return Scene(self.pos.copy(), self.vel.copy(), self.mass.copy(), self.geom.copy(),
                     self.fixed.copy(), self.family.copy(), dict(self.params), self.name,
                     None if self.gamma is None else self.gamma.copy(),
                     None if self.bilateral is None else list(self.bilateral))


def default_params(**kw) -> dict:
    """Defaults of the reference: h = 1e-3, mu = 0.25 (System.cu:62-72),
    envelope 0.001 (CollisionDetector.cu:512), APGD tolerance 1e-4 and
    maxIterations 100000 (APGD.cu:10-11), warm start off (APGD.cu:14)."""
    p = dict(h=1e-3, mu=0.25, gravity=(0.0, -9.81, 0.0), envelope=1e-3, tolerance=1e-4,
             max_iterations=100000, warm_start=0, max_backtracks=4096)
    p.update(kw)
    return p


def _assemble(boxes, spheres_pos, spheres_r, rho, params, name, spheres_vel=None):
    nbx = len(boxes)
    ns = spheres_pos.shape[0]
    nb = nbx + ns
    pos = np.zeros((nb, 3))
    geom = np.zeros((nb, 3))
    mass = np.ones(nb)
    fixed = np.zeros(nb, dtype=np.int32)
    for i, (c, he, fx) in enumerate(boxes):
        pos[i] = c
        geom[i] = he
        fixed[i] = 1 if fx else 0
    pos[nbx:] = spheres_pos
    geom[nbx:, 0] = spheres_r
    mass[nbx:] = rho * 4.0 / 3.0 * math.pi * spheres_r ** 3
    vel = np.zeros((nb, 3))
    if spheres_vel is not None:
        vel[nbx:] = spheres_vel
    family = np.full(nb, -1, dtype=np.int32)
    return Scene(pos, vel, mass, geom, fixed, family, params, name)


def open_box(inner_x, inner_y, height, thick=0.1, cx=0.0, cy=0.0):
    """Floor + 4 walls, all fixed; floor top at z = 0 and interior
    [cx - inner_x/2, cx + inner_x/2] x [cy - inner_y/2, cy + inner_y/2]."""
    t = 0.5 * thick
    hx, hy = 0.5 * inner_x, 0.5 * inner_y
    return [
        ((cx, cy, -t), (hx + thick, hy + thick, t), True),
        ((cx - hx - t, cy, 0.5 * height), (t, hy + thick, 0.5 * height), True),
        ((cx + hx + t, cy, 0.5 * height), (t, hy + thick, 0.5 * height), True),
        ((cx, cy - hy - t, 0.5 * height), (hx, t, 0.5 * height), True),
        ((cx, cy + hy + t, 0.5 * height), (hx, t, 0.5 * height), True),
    ]


def settling_box(seed=0, n_side=10, radius=0.05, spacing=0.11, jitter=0.005, rho=2600.0,
                 mu=0.25, h=1e-3, tolerance=1e-4, max_iterations=1000, warm_start=1) -> Scene:
    rng = np.random.default_rng(seed)
    idx = np.arange(n_side)
    off = -0.5 * spacing * (n_side - 1)
    gx, gy, gz = np.meshgrid(idx, idx, idx, indexing="ij")
    pos = np.stack([off + spacing * gx.ravel(), off + spacing * gy.ravel(),
                    radius + 0.01 + spacing * gz.ravel()], axis=1)
    pos += rng.uniform(-jitter, jitter, size=pos.shape)
    r = np.full(pos.shape[0], radius)
    inner = 1.2 * (n_side / 10.0)
    boxes = open_box(inner, inner, 1.5 * (n_side / 10.0))
    params = default_params(h=h, mu=mu, gravity=(0.0, 0.0, -G), tolerance=tolerance,
                            max_iterations=max_iterations, warm_start=warm_start)
    return _assemble(boxes, pos, r, rho, params, f"settling_box_{pos.shape[0]}")


def _rsa_column(rng, n, rmin, rmax, lx, ly, z0, fill=0.30, batch=16384):
    """Random sequential addition: spheres are drawn uniformly in the column;
    a draw is rejected when it overlaps an accepted sphere or an earlier draw of
    its batch.  Radii are drawn with the positions, so the accepted radii keep
    the U[rmin, rmax] law only approximately (small spheres fit more often)."""
    from scipy.spatial import cKDTree

    mean_v = 4.0 / 3.0 * math.pi * (rmax ** 4 - rmin ** 4) / (4.0 * (rmax - rmin))
    height = n * mean_v / (fill * lx * ly) + 2 * rmax
    P = np.zeros((0, 3))
    R = np.zeros(0)
    while P.shape[0] < n:
        k = batch
        r = rng.uniform(rmin, rmax, size=k)
        p = np.stack([rng.uniform(r, lx - r), rng.uniform(r, ly - r),
                      rng.uniform(r, height - r)], axis=1)
        ok = np.ones(k, dtype=bool)
        if P.shape[0]:
            tree = cKDTree(P)
            d, idx = tree.query(p, k=24, distance_upper_bound=2 * rmax)
            valid = np.isfinite(d)
            idc = np.where(valid, idx, 0)
            ok &= ~np.any(valid & (d <= R[idc] + r[:, None]), axis=1)
        cand = np.nonzero(ok)[0]
        if cand.size > 1:
            pairs = cKDTree(p[cand]).query_pairs(2 * rmax, output_type="ndarray")
            if pairs.size:
                i, j = pairs[:, 0], pairs[:, 1]
                dd = np.linalg.norm(p[cand[i]] - p[cand[j]], axis=1)
                hit = dd <= r[cand[i]] + r[cand[j]]
                later = np.maximum(i[hit], j[hit])
                keep = np.ones(cand.size, dtype=bool)
                keep[later] = False
                cand = cand[keep]
        take = cand[: n - P.shape[0]]
        P = np.concatenate([P, p[take]])
        R = np.concatenate([R, r[take]])
    P = P.copy()
    P[:, 0] -= 0.5 * lx
    P[:, 1] -= 0.5 * ly
    P[:, 2] += z0
    return P, R, height


def poured_column(seed=1, n=200_000, rmin=0.004, rmax=0.006, rho=2500.0, mu=0.3, h=5e-4,
                  lx=0.4, ly=0.4, tolerance=1e-4, max_iterations=500, warm_start=1,
                  fill=0.30) -> Scene:
    rng = np.random.default_rng(seed)
    P, R, height = _rsa_column(rng, n, rmin, rmax, lx, ly, 0.0, fill=fill)
    boxes = open_box(lx, ly, height + 0.1, thick=0.05)
    params = default_params(h=h, mu=mu, gravity=(0.0, 0.0, -G), tolerance=tolerance,
                            max_iterations=max_iterations, warm_start=warm_start)
    return _assemble(boxes, P, R, rho, params, f"poured_column_{n}")


def lattice_container(rng, n, rmin=0.004, rmax=0.006, rho=2500.0, mu=None, h=1e-3,
                      tolerance=1e-4, max_iterations=500, warm_start=1, name="batch"):
    """One settling scene of n spheres: square floor of side ~ cbrt(n) * 2.2 r_max,
    walls twice the fill height, spheres on a jittered lattice of spacing 2.2 r_max."""
    if mu is None:
        mu = float(rng.uniform(0.1, 0.5))
    s = 2.2 * rmax
    side_n = max(1, int(round(n ** (1.0 / 3.0))))
    layers = int(math.ceil(n / float(side_n * side_n)))
    inner = side_n * s
    fill_h = layers * s
    gi = np.arange(n)
    ix, iy, iz = gi % side_n, (gi // side_n) % side_n, gi // (side_n * side_n)
    jit = 0.5 * (s - 2 * rmax) * 0.9
    pos = np.stack([(ix + 0.5) * s - 0.5 * inner, (iy + 0.5) * s - 0.5 * inner,
                    (iz + 0.5) * s], axis=1) + rng.uniform(-jit, jit, size=(n, 3))
    r = rng.uniform(rmin, rmax, size=n)
    boxes = open_box(inner, inner, 2.0 * fill_h + s, thick=0.02)
    params = default_params(h=h, mu=mu, gravity=(0.0, 0.0, -G), tolerance=tolerance,
                            max_iterations=max_iterations, warm_start=warm_start)
    return _assemble(boxes, pos, r, rho, params, name)


def batch_scenes(seed=3, count=512, nmin=100, nmax=20000, **kw):
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=count)).astype(np.int64)
    return [lattice_container(rng, int(n), name=f"batch_{i}_{int(n)}", **kw)
            for i, n in enumerate(ns)]


def ball_on_ground(h=1e-2, tolerance=1e-5, warm_start=0, latforce=0.0) -> Scene:
    """models/test_oneBall.cu:240-283: fixed unit box at y = -1, unit ball
    (mass 1) at y = 1, gravity (latForce, -9.81, 0), h = 1e-2."""
    pos = np.array([[0.0, -1.0, 0.0], [0.0, 1.0, 0.0]])
    geom = np.array([[1.0, 1.0, 1.0], [1.0, 0.0, 0.0]])
    params = default_params(h=h, tolerance=tolerance, warm_start=warm_start,
                            gravity=(latforce, -9.81, 0.0), max_iterations=100000)
    return Scene(pos, np.zeros((2, 3)), np.ones(2), geom, np.array([1, 0], dtype=np.int32),
                 np.full(2, -1, dtype=np.int32), params, "ball_on_ground")


def sphere_stack(n=5, radius=0.05, rho=2600.0, mu=0.25, h=1e-3, tolerance=1e-8,
                 max_iterations=20000, warm_start=1, overlap=0.0) -> Scene:
    """n equal spheres stacked on one vertical line on a fixed floor, each
    touching the one below (gap -overlap): n contacts in a chain, every
    normal exactly vertical.  The contact impulses are unique (the solve is
    determinate): at rest the k-th contact from the top carries k m g h."""
    z = radius - overlap + np.arange(n) * (2.0 * radius - overlap)
    pos = np.stack([np.zeros(n), np.zeros(n), z], axis=1)
    boxes = [((0.0, 0.0, -0.05), (0.5, 0.5, 0.05), True)]
    params = default_params(h=h, mu=mu, gravity=(0.0, 0.0, -G), tolerance=tolerance,
                            max_iterations=max_iterations, warm_start=warm_start)
    return _assemble(boxes, pos, np.full(n, radius), rho, params, f"stack_{n}")


def random_cluster(seed, n=40, box=True, radius=0.05, mu=0.25, h=1e-3, warm_start=1,
                   max_iterations=400, tolerance=1e-6) -> Scene:
    """Small parity-test scene: spheres on a jittered cubic lattice whose
    spacing equals the largest diameter, so neighbours range from slightly
    overlapping through inside the envelope to just separated; the lowest
    layer rests on a fixed floor inside fixed walls; random initial velocities."""
    rng = np.random.default_rng(seed)
    side = max(2, int(math.ceil(n ** (1.0 / 3.0))))
    s = 2.0 * radius
    gi = np.arange(n)
    ix, iy, iz = gi % side, (gi // side) % side, gi // (side * side)
    pos = np.stack([(ix - 0.5 * (side - 1)) * s, (iy - 0.5 * (side - 1)) * s, radius + iz * s],
                   axis=1)
    pos += rng.uniform(-0.0015, 0.0015, size=pos.shape)
    r = rng.uniform(0.97 * radius, radius, size=n)
    inner = side * s + 0.004
    boxes = open_box(inner, inner, (side + 2) * s, thick=0.1) if box else []
    params = default_params(h=h, mu=mu, gravity=(0.0, 0.0, -G), tolerance=tolerance,
                            max_iterations=max_iterations, warm_start=warm_start)
    vel = rng.normal(0.0, 0.05, size=(n, 3))
    return _assemble(boxes, pos, r, 2600.0, params, f"cluster_{seed}_{n}", spheres_vel=vel)


def free_balls(n=2, spacing=0.5, radius=0.05, h=1e-3, warm_start=1, vel=None,
               tolerance=1e-10, max_iterations=2000) -> Scene:
    """n unit-density spheres far apart in free flight under gravity -z (no
    contacts ever): a scene whose only constraints are bilateral rows."""
    pos = np.zeros((n, 3))
    pos[:, 0] = spacing * np.arange(n)
    pos[:, 2] = 1.0
    params = default_params(h=h, gravity=(0.0, 0.0, -G), tolerance=tolerance,
                            max_iterations=max_iterations, warm_start=warm_start)
    sc = _assemble([], pos, np.full(n, radius), 1000.0, params, f"free_balls_{n}",
                   spheres_vel=None if vel is None else np.asarray(vel, dtype=np.float64))
    return sc


def crowd(n_around, seed=5, radius=0.05, max_iterations=50) -> Scene:
    """Sphere 0 with n_around equal spheres overlapping it, all with larger
    ids (centres 0.5 to 1.5 radii from its centre, random directions), in
    free space under gravity -z: one free body in contact with n_around
    others, and the others with some of each other."""
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n_around, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    c = np.array([0.0, 0.0, 1.0])
    pos = np.concatenate([c[None], c + d * radius * rng.uniform(0.5, 1.5, size=(n_around, 1))])
    params = default_params(gravity=(0.0, 0.0, -G), max_iterations=max_iterations)
    return _assemble([], pos, np.full(n_around + 1, radius), 2600.0, params,
                     f"crowd_{n_around}")


def raspberry(n, big=1.0, small=0.015, overlap=5e-4, ballast=0, max_iterations=50) -> Scene:
    """One sphere of radius `big` (body 0) with n spheres of radius `small` on
    its surface (a Fibonacci lattice, each overlapping it by `overlap`), in
    free space without gravity: body 0 has n contact partners, all with
    larger ids; the small spheres are too far apart to touch one another.
    With ballast = m > 0, m spheres of radius big / 3 on a lattice 1 m apart,
    20 m away and touching nothing, raise the median radius so that the big
    sphere goes through the uniform grid and the sphere pair kernels (a
    sphere above four times the median radius is paired against every body
    of its scene instead)."""
    i = np.arange(n) + 0.5
    z = 1.0 - 2.0 * i / n
    rho = np.sqrt(1.0 - z * z)
    phi = i * math.pi * (3.0 - math.sqrt(5.0))
    d = big + small - overlap
    pos = [np.zeros((1, 3)), d * np.stack([rho * np.cos(phi), rho * np.sin(phi), z], axis=1)]
    r = [np.array([big]), np.full(n, small)]
    if ballast:
        k = int(math.ceil(ballast ** (1.0 / 3.0)))
        g = np.stack(np.meshgrid(np.arange(k), np.arange(k), np.arange(k), indexing="ij"),
                     axis=-1).reshape(-1, 3)[:ballast]
        pos.append(20.0 + g.astype(np.float64))
        r.append(np.full(ballast, big / 3.0))
    pos = np.concatenate(pos)
    r = np.concatenate(r)
    params = default_params(gravity=(0.0, 0.0, 0.0), max_iterations=max_iterations)
    return _assemble([], pos, r, 2600.0, params, f"raspberry_{n}")


def bilateral_cluster(seed, n=64, warm_start=1, h=1e-3, max_iterations=400,
                      tolerance=1e-6) -> Scene:
    """random_cluster with bilateral rows (System::addBilateralConstraintDOF,
    as the reference drivers pin DOFs): the first sphere held in x (in z it
    could start inside the floor, an infeasible pair of rows), the second
    and third spheres' y coupled (a two-DOF row drives y_A - y_B to 0; these
    two differ by the lattice jitter only), the fourth sphere's y moved at
    0.1 m/s from t = 2 h on, and a row on a fixed box's DOF (a zero row of N)."""
    sc = random_cluster(seed, n=n, warm_start=warm_start, h=h,
                        max_iterations=max_iterations, tolerance=tolerance)
    s0 = int(np.argmax(sc.fixed == 0))  # first sphere (the boxes come first)
    sc.bilateral = [(3 * s0, -1, 0.0, 0.0),
                    (3 * (s0 + 1) + 1, 3 * (s0 + 2) + 1, 0.0, 0.0),
                    (3 * (s0 + 3) + 1, -1, 0.1, 2 * h),
                    (0, -1, 0.0, 0.0)]
    sc.name = f"bilateral_{seed}_{n}"
    return sc
