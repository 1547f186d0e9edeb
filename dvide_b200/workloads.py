"""Benchmark workloads built from the seeded scenes of scenes.py.

``column_settled()`` is the 200,000-sphere column (r ~ U[0.004, 0.006] m,
rho = 2500, mu = 0.3, h = 5e-4, APGD tolerance 1e-4, at most 500 iterations,
warm start) after it has been poured from its random non-overlapping packing
and has come to rest: about 7.3e5 contacts per step.  The rest state is kept
in data/column_settled.npz (float32 positions and radii; velocities zero) so
that every benchmark arm starts from the same input.  make_column_settled()
regenerates it: random sequential addition (scenes.poured_column, seed 1),
then 4,000 steps of the contact step itself with a loose solve (tolerance
1e-3, 50 iterations) until the kinetic energy is ~1e-2 J.
"""
from __future__ import annotations

import os

import numpy as np

from . import scenes

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
COLUMN_FILE = os.path.join(DATA, "column_settled.npz")

COLUMN_PARAMS = dict(h=5e-4, mu=0.3, tolerance=1e-4, max_iterations=500, warm_start=1)


def _column_scene(pos, r, wall_height):
    boxes = scenes.open_box(0.4, 0.4, wall_height, thick=0.05)
    params = scenes.default_params(gravity=(0.0, 0.0, -scenes.G), **COLUMN_PARAMS)
    sc = scenes._assemble(boxes, pos, r, 2500.0, params, "column_settled")
    return sc


def column_settled(path=COLUMN_FILE) -> scenes.Scene:
    d = np.load(path)
    pos = d["pos"].astype(np.float64)
    r = d["radius"].astype(np.float64)
    return _column_scene(pos, r, float(d["wall_height"]))


def make_column_settled(path=COLUMN_FILE, steps=4000, n=200_000, seed=1):
    from . import _native as N
    col = scenes.poured_column(seed=seed, n=n)
    wall_h = 2.0 * col.pos[1, 2]  # the walls of scenes.poured_column
    sc = _column_scene(col.pos[5:], col.geom[5:, 0], wall_h)
    g = N.NativeScene.from_scene(sc, tolerance=1e-3, max_iterations=50)
    g.step(steps)
    p, _ = g.state()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, pos=p[5:].astype(np.float32),
                        radius=sc.geom[5:, 0].astype(np.float32),
                        wall_height=np.float64(wall_h))
    return path


def settling_box():
    """1,000-sphere settling box (the CPU-runnable configuration)."""
    return scenes.settling_box()
