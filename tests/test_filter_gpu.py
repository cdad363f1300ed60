"""Contact de-duplication on the GPU (delta_filter_new_contacts, delta_filter_old_contacts)
against the oracle (oracle/delta_oracle.c, pinned to filter.cpp): keep flags bit-exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _contacts(x, master, slave, capacity=None):
    import torch

    from delta_b200.detection import Contacts

    n = x.shape[1]
    c = Contacts(capacity or max(n, 1))
    c.x[:, :n] = torch.from_numpy(np.ascontiguousarray(x))
    c.master[:n] = torch.from_numpy(np.asarray(master, np.int32))
    c.slave[:n] = torch.from_numpy(np.asarray(slave, np.int32))
    for name in ("normal", "P", "Q"):
        getattr(c, name).zero_()
    for name in ("depth", "eps_total", "tri_a", "tri_b", "penetration", "friction"):
        getattr(c, name).zero_()
    c.count = n
    return c


def _runs(rng, sizes, scale=1e-3):
    steps = np.array([0.0, 5e-5, 9.99e-5, 1e-4, 2e-4])
    n = int(sum(sizes))
    x = rng.uniform(0, scale, (3, n // 4 + 1))[:, rng.integers(0, n // 4 + 1, n)] + rng.choice(steps, (3, n))
    master = np.repeat(np.arange(len(sizes), dtype=np.int32) // 3, sizes)
    slave = np.repeat(np.arange(len(sizes), dtype=np.int32), sizes)
    return x, master, slave


@pytest.mark.parametrize("seed", [0, 1])
def test_filter_new_matches_oracle(ctx, oracle, seed):
    from delta_b200.detection import filter_new_mask

    rng = np.random.default_rng(seed)
    sizes = list(rng.integers(1, 60, 500)) + [1500, 1, 2, 700]  # many runs, two long ones
    x, m, s = _runs(rng, sizes)
    c = _contacts(x, m, s, capacity=x.shape[1] + 37)  # ld = capacity > n
    keep = filter_new_mask(ctx, c).cpu().numpy()
    assert np.array_equal(keep, oracle.filter_new(x, m, s))
    assert 0 < keep.sum() < keep.size


def test_filter_old_matches_oracle(ctx, oracle):
    from delta_b200.detection import filter_old_mask

    rng = np.random.default_rng(5)
    xs, ms, ss = _runs(rng, list(rng.integers(1, 40, 300)))
    xn, mn, sn = _runs(rng, list(rng.integers(1, 40, 300)))
    perm = rng.permutation(xs.shape[1])  # stored contacts in any order
    xs, ms, ss = xs[:, perm], ms[perm], ss[perm]
    keep = filter_old_mask(ctx, _contacts(xs, ms, ss), _contacts(xn, mn, sn)).cpu().numpy()
    assert np.array_equal(keep, oracle.filter_old(xs, ms, ss, xn, mn, sn))
    assert 0 < keep.sum() < keep.size


def test_filter_edge_cases(ctx, oracle):
    from delta_b200.detection import filter_new_mask, filter_old_mask

    x = np.array([[0.0, 0.6e-4, 1.2e-4, 0.0], [0, 0, 0, 0], [0, 0, 0, 0]])
    m = np.zeros(4, np.int32)
    s = np.array([0, 0, 0, 1], np.int32)
    assert list(filter_new_mask(ctx, _contacts(x, m, s)).cpu().numpy()) == [1, 0, 1, 1]
    empty = _contacts(np.zeros((3, 0)), [], [])
    assert filter_new_mask(ctx, empty).numel() == 0
    # no stored contacts: everything stays
    keep = filter_old_mask(ctx, empty, _contacts(x, m, s)).cpu().numpy()
    assert list(keep) == [1, 1, 1, 1]


def test_filter_on_detected_contacts(ctx, oracle):
    """On the contacts the detector returns for overlapping perturbed spheres (the runs are
    the particle pairs), large halo so that neighbouring triangle pairs give near contacts."""
    from delta_b200.detection import Meshes, detect, filterNewContacts
    from delta_b200.scenarios import sphere_mesh

    rng = np.random.default_rng(11)
    bodies = []
    for k, nt in enumerate((80, 160, 80, 320)):
        V, F = sphere_mesh(nt, rng, 0.05, (0.9, 1.1))
        bodies.append((V[F].reshape(-1, 3) + np.array([0.09 * k, 0.0, 0.0])).T.copy())
    m = Meshes.from_bodies(bodies, np.full(4, 0.01), np.zeros(4, np.uint8), np.arange(4))
    contacts, _ = detect(ctx, 0, m, [0, 1, 2, 0], [1, 2, 3, 2])
    arr = contacts.to_numpy()
    keep_ref = oracle.filter_new(np.ascontiguousarray(arr["x"].T), arr["master"], arr["slave"])
    out = filterNewContacts(ctx, contacts)
    assert 0 < out.count == int(keep_ref.sum()) < contacts.count
    kept = out.to_numpy()
    assert np.array_equal(kept["x"], arr["x"][keep_ref.astype(bool)])
    assert np.array_equal(kept["tri_b"], arr["tri_b"][keep_ref.astype(bool)])
