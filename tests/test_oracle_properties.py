"""Property-based checks (hypothesis) of the oracle's building blocks, which
the GPU path matches bit for bit:
- the friction-cone projection (APGD.cu:47-78) is the Euclidean projection
  onto K = {|g_t| <= mu g_n} (Moreau: P(x) in K, x - P(x) in the polar cone,
  the two orthogonal; P idempotent), except the reference's branch that sends
  a point outside K with |g_n| < 1e-14 to zero (APGD.cu:63);
- the matrix-free Schur product N = D Minv D^T (APGD.cu:81-87) is symmetric,
  positive semidefinite and linear on random clusters' contacts;
- the tangent frame (System.cu:753-762) is orthonormal to float precision;
- the ordered sum stays within the rounding bound of the exact sum."""
import math

import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

from dvide_b200 import scenes

coord = st.floats(min_value=-1e3, max_value=1e3, allow_nan=False, allow_infinity=False)
mus = st.one_of(st.just(0.0), st.floats(min_value=1e-3, max_value=2.0))


@settings(max_examples=400, deadline=None, derandomize=True, database=None)
@given(x=st.tuples(coord, coord, coord), mu=mus)
def test_cone_projection_is_the_projection(oracle_mod, x, mu):
    x = np.array(x)
    p = oracle_mod.project(x, mu)
    scale = max(1.0, np.abs(x).max())
    gt = math.sqrt(x[1] * x[1] + x[2] * x[2])  # as APGD.cu:54 (it may underflow)
    if mu > 0 and abs(x[0]) < 1e-14 and not gt < mu * x[0]:
        # APGD.cu:63: treated as the polar cone's
        assert (p == 0.0).all()
        return
    pt = math.hypot(p[1], p[2])
    eps = 1e-12 * scale
    # P(x) in K
    if mu == 0:
        assert p[1] == 0.0 and p[2] == 0.0 and p[0] >= 0.0
    else:
        assert pt <= mu * p[0] * (1 + 1e-12) + eps
    # x - P(x) in the polar cone, orthogonal to P(x)
    d = x - p
    if mu == 0:
        assert d[0] <= eps
    else:
        assert math.hypot(d[1], d[2]) * mu <= -d[0] * (1 + 1e-9) + eps
    assert abs(float(d @ p)) <= 1e-12 * scale * scale
    # idempotent (a point on K's edge may move by rounding)
    q = oracle_mod.project(p, mu)
    assert np.abs(q - p).max() <= eps


@settings(max_examples=25, deadline=None, derandomize=True, database=None)
@given(seed=st.integers(0, 200), vseed=st.integers(0, 2**31 - 1),
       a=st.floats(-10, 10), b=st.floats(-10, 10))
def test_schur_product_symmetric_psd_linear(oracle_mod, seed, vseed, a, b):
    sc = scenes.random_cluster(seed, n=25)
    o = oracle_mod.OracleScene(sc)
    o.collide()
    ia, ib, _, _ = o.contacts()
    if ia.size == 0:
        return
    F = o.frames()
    minv = np.repeat(np.where(sc.fixed == 1, 0.0, 1.0 / sc.mass), 3)
    rng = np.random.default_rng(vseed)
    x = rng.standard_normal(3 * ia.size)
    y = rng.standard_normal(3 * ia.size)

    def N(v):
        return oracle_mod.schur(sc.nb, ia, ib, F, minv, v)

    Nx, Ny = N(x), N(y)
    big = max(np.abs(Nx).max(), np.abs(Ny).max(), 1e-300)
    n = float(np.linalg.norm(x) * np.linalg.norm(y))
    assert abs(float(y @ Nx) - float(Ny @ x)) <= 1e-12 * big * n
    assert float(x @ Nx) >= -1e-12 * big * float(x @ x)
    lin = N(a * x + b * y)
    assert np.allclose(lin, a * Nx + b * Ny, rtol=0, atol=1e-12 * big * (abs(a) + abs(b) + 1))


unit = st.floats(min_value=-1.0, max_value=1.0, allow_nan=False)


@settings(max_examples=300, deadline=None, derandomize=True, database=None)
@given(n=st.tuples(unit, unit, unit))
def test_frame_orthonormal_to_float_precision(oracle_mod, n):
    n = np.array(n)
    norm = np.linalg.norm(n)
    if norm < 1e-3:
        return
    n = n / norm
    u, v = oracle_mod.frame(n)
    if 0 < abs(n[2]) < 1e-12:
        # -n_x / n_z overflows the float dot product of the normalisation when
        # |n_z| is below ~5e-20 |n_x| (u collapses to 0, as in the reference);
        # a contact normal's nonzero n_z is never that small (positions differ
        # by at least one ulp)
        return
    tol = 1e-6  # the frame is normalised with float square roots and divisions
    assert abs(np.linalg.norm(u) - 1) < tol and abs(np.linalg.norm(v) - 1) < tol
    assert abs(u @ n) < tol and abs(v @ n) < tol and abs(u @ v) < tol


@settings(max_examples=200, deadline=None, derandomize=True, database=None)
@given(v=st.lists(st.floats(-1e6, 1e6, allow_nan=False), min_size=0, max_size=3000))
def test_ordered_sum_within_rounding_bound(oracle_mod, v):
    s = oracle_mod.ordered_sum(v)
    exact = math.fsum(v)
    bound = (len(v) + 1) * 2.0 ** -52 * math.fsum(abs(x) for x in v)
    assert abs(s - exact) <= bound
