"""Property checks of the pair solvers (the reference pins no narrowphase results, so
these complement the oracle comparisons): on separated pairs bfSolver's distance equals
the separation the generator built, lies below every sampled point-pair distance, and is
unchanged by swapping A and B or by a rigid motion, up to FP64 rounding.  Intersecting
pairs break the sampled bound, as the reference's bfSolver does not detect intersections
(bf.cpp:359-407 is dead code)."""
import numpy as np
import pytest

ABS = 4e-15  # FP64 rounding at unit-size coordinates (observed at most 6e-16)


@pytest.fixture(scope="module")
def workload(oracle):
    from delta_b200.scenarios import narrowphase_pairs

    a, b, d, cls = narrowphase_pairs(3000, seed=77)
    _, _, bd, _ = oracle.pairs(0, a, b)
    return a, b, d, cls, bd


def _separated(cls):
    from delta_b200.scenarios import INTERSECTING

    return cls != INTERSECTING


def _sampled_min(a, b, levels=8):
    g = [(i, j) for i in range(levels + 1) for j in range(levels + 1 - i)]
    W = np.array([[1 - (i + j) / levels, i / levels, j / levels] for i, j in g])
    PA = np.einsum("kv,nvc->nkc", W, a.T.reshape(-1, 3, 3))
    PB = np.einsum("kv,nvc->nkc", W, b.T.reshape(-1, 3, 3))
    return np.sqrt(((PA[:, :, None, :] - PB[:, None, :, :]) ** 2).sum(-1)).min((1, 2))


def test_bf_equals_constructed_separation(workload):
    a, b, d, cls, bd = workload
    s = _separated(cls)
    assert np.all(np.abs(bd[s] - d[s]) <= ABS)


def test_bf_below_sampled_distances_and_intersections_missed(workload):
    a, b, d, cls, bd = workload
    s = _separated(cls)
    dm = _sampled_min(a, b)
    assert np.all(bd[s] <= dm[s] * (1 + 1e-12))
    assert np.any(bd[~s] > dm[~s] + 1e-9)  # reference behaviour: intersections not seen


def test_bf_symmetric_under_swap(oracle, workload):
    a, b, d, cls, bd = workload
    _, _, bd2, _ = oracle.pairs(0, b, a)
    s = _separated(cls)
    assert np.all(np.abs(bd2[s] - bd[s]) <= ABS)


def test_bf_invariant_under_rigid_motion(oracle, workload):
    a, b, d, cls, bd = workload
    rng = np.random.default_rng(1)
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    t = rng.normal(size=3)
    A = a.T.reshape(-1, 3, 3) @ q.T + t
    B = b.T.reshape(-1, 3, 3) @ q.T + t
    _, _, bd3, _ = oracle.pairs(0, np.ascontiguousarray(A.reshape(-1, 9).T), np.ascontiguousarray(B.reshape(-1, 9).T))
    s = _separated(cls)
    assert np.all(np.abs(bd3[s] - bd[s]) <= ABS)


@pytest.mark.gpu
def test_gpu_solvers_keep_the_properties(ctx, workload):
    """bf_cert (bit-exact) and the learned hybrid (within 1e-6) on the GPU: the constructed
    separation of separated pairs, and symmetry under swapping A and B."""
    import torch

    from delta_b200.learned import learned_pairs
    from delta_b200.narrowphase import pairs_device

    a, b, d, cls, bd = workload
    s = _separated(cls)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    cert = pairs_device(ctx, 5, da, db)[2]
    ctx.synchronize()
    cert = cert.cpu().numpy()
    assert np.array_equal(cert, bd, equal_nan=True)
    for x, y in ((da, db), (db, da)):
        ld = learned_pairs(ctx, None, x, y, sweeps=2, features=3)[2]
        ctx.synchronize()
        ld = ld.cpu().numpy()
        assert np.all(np.abs(ld[s] - d[s]) <= 1e-6 * d[s] + ABS)
