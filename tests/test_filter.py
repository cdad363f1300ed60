"""Contact de-duplication (filter.cpp): the oracle against the reference's own functions
(oracle/_ref) on the CPU, including the edge cases the greedy rule has."""
import numpy as np
import pytest

from oracle.oracle import Oracle, Reference

pytestmark = pytest.mark.skipif(not Reference.available(), reason="reference library not built")


def clustered(n, rng, scale=1e-3, steps=(0.0, 5e-5, 9.99e-5, 2e-4)):
    """Points on a coarse lattice of offsets below and above eps = 1e-4."""
    base = rng.uniform(0, scale, (3, n // 4 + 1))[:, rng.integers(0, n // 4 + 1, n)]
    return base + rng.choice(np.asarray(steps), (3, n))


@pytest.mark.parametrize("seed", range(5))
def test_filter_new_oracle_equals_reference(seed):
    rng = np.random.default_rng(seed)
    x = clustered(400, rng)
    z = np.zeros(400, np.int32)
    assert np.array_equal(Oracle().filter_new(x, z, z), Reference().filter_new(x))


@pytest.mark.parametrize("seed", range(5))
def test_filter_old_oracle_equals_reference(seed):
    rng = np.random.default_rng(100 + seed)
    xs, xn = clustered(150, rng), clustered(250, rng)
    zs, zn = np.zeros(150, np.int32), np.zeros(250, np.int32)
    assert np.array_equal(Oracle().filter_old(xs, zs, zs, xn, zn, zn), Reference().filter_old(xs, xn))


def test_filter_new_edge_cases():
    o, r = Oracle(), Reference()
    z = lambda n: np.zeros(n, np.int32)  # noqa: E731
    # chain: b near a (dropped), c near b but not a: kept, because dropped contacts drop nothing
    x = np.array([[0.0, 0.6e-4, 1.2e-4], [0, 0, 0], [0, 0, 0]])
    assert list(o.filter_new(x, z(3), z(3))) == [1, 0, 1] == list(r.filter_new(x))
    # exact duplicates: the first stays
    x = np.zeros((3, 4))
    assert list(o.filter_new(x, z(4), z(4))) == [1, 0, 0, 0] == list(r.filter_new(x))
    # a difference of exactly eps is not near (strict <)
    x = np.array([[0.0, 1e-4], [0, 0], [0, 0]])
    assert list(o.filter_new(x, z(2), z(2), eps=1e-4)) == list(r.filter_new(x))
    # near on two coordinates only: kept
    x = np.array([[0.0, 0.0], [0.0, 0.0], [0.0, 5e-4]])
    assert list(o.filter_new(x, z(2), z(2))) == [1, 1] == list(r.filter_new(x))
    # empty and single
    assert o.filter_new(np.zeros((3, 0)), z(0), z(0)).size == 0
    assert list(o.filter_new(np.ones((3, 1)), z(1), z(1))) == [1]


def test_filter_runs_are_independent():
    """Per (master, slave) run, the oracle equals the reference applied to that run alone."""
    rng = np.random.default_rng(7)
    sizes = [1, 5, 40, 3, 120, 2]
    x = clustered(sum(sizes), rng)
    master = np.repeat(np.arange(len(sizes), dtype=np.int32) // 2, sizes)
    slave = np.repeat(np.arange(len(sizes), dtype=np.int32), sizes)
    keep = Oracle().filter_new(x, master, slave)
    s = 0
    for k in sizes:
        assert np.array_equal(keep[s:s + k], Reference().filter_new(x[:, s:s + k]))
        s += k
