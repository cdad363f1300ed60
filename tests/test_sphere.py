"""Sphere model (sphere.cpp, point.cpp): the oracle against the reference's own functions on
the CPU, bit for bit."""
import numpy as np
import pytest

from oracle.oracle import CONTACT_DTYPE, Oracle, Reference

pytestmark = pytest.mark.skipif(not Reference.available(), reason="reference library not built")
FIELDS = [f for f in CONTACT_DTYPE.names if f not in ("tri_a", "tri_b")]


def _same(a, b):
    return len(a) == len(b) and all(np.array_equal(a[f], b[f], equal_nan=True) for f in FIELDS)


def test_pt_oracle_equals_reference():
    o, r = Oracle(), Reference()
    rng = np.random.default_rng(0)
    for _ in range(5000):
        T = rng.normal(size=(3, 3))
        c = rng.normal(size=3) * 2
        d1, q1 = o.pt(T[0], T[1], T[2], c)
        d2, q2 = r.pt(T[0], T[1], T[2], c)
        assert d1 == d2 and np.array_equal(q1, q2)
    # degenerate triangle (zero area): same NaN/inf behaviour
    T = np.zeros((3, 3))
    d1, q1 = o.pt(T[0], T[1], T[2], np.ones(3))
    d2, q2 = r.pt(T[0], T[1], T[2], np.ones(3))
    assert np.array_equal(np.array([d1, *q1]), np.array([d2, *q2]), equal_nan=True)


def test_sphere_oracle_equals_reference():
    o, r = Oracle(), Reference()
    rng = np.random.default_rng(1)
    hits = 0
    for _ in range(2000):
        cA = rng.normal(size=3) * 0.01
        cB = cA + rng.normal(size=3) * 0.01
        args = (cA, rng.uniform(0.005, 0.015), 1e-3, rng.integers(0, 2), 3, cB, rng.uniform(0.005, 0.015), 2e-3,
                rng.integers(0, 2), 7)
        a, b = o.sphere(*args), r.sphere(*args)
        hits += len(a)
        assert _same(a, b)
    assert hits > 100


@pytest.mark.parametrize("ba", [0, 1])
def test_sphere_mesh_oracle_equals_reference(ba):
    from delta_b200.scenarios import sphere_mesh

    o, r = Oracle(), Reference()
    rng = np.random.default_rng(2 + ba)
    V, F = sphere_mesh(80, rng, 0.05, (0.9, 1.1))
    M = V[F].reshape(-1, 3).T.copy()
    hits = 0
    for _ in range(150):
        c = rng.normal(size=3) * 0.03
        d = rng.uniform(0.01, 0.06)
        a = o.sphere_mesh(ba, c, d, 1e-3, 1, 4, M, 80, 2e-3, 1, 9)
        b = r.sphere_mesh(ba, c, d, 1e-3, 1, 4, M, 80, 2e-3, 1, 9)
        hits += len(a)
        assert _same(a, b)
    assert hits > 50


def test_sphere_overlay_oracle_equals_reference():
    o, r = Oracle(), Reference()
    rng = np.random.default_rng(4)
    for _ in range(5000):
        cA, cB = rng.normal(size=3), rng.normal(size=3)
        rA, rB = rng.uniform(0, 1.5, 2)
        assert o.sphere_overlay(cA, rA, cB, rB) == r.sphere_overlay(cA, rA, cB, rB)
