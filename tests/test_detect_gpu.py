"""Particle-pair drivers on the GPU against the oracle (bit for bit in FP64)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["x", "normal", "depth", "P", "Q", "friction", "eps_total", "master", "slave", "penetration", "tri_a",
          "tri_b"]


def _scene(seed, sizes=(20, 40, 80, 20, 40), eps=0.003):
    """Bodies in a row, neighbours overlapping slightly; candidate pairs (i, i+1) and (i, i+2)."""
    from delta_b200.scenarios import sphere_mesh

    rng = np.random.default_rng(seed)
    bodies = []
    for k, nt in enumerate(sizes):
        V, F = sphere_mesh(nt, rng, 0.05, (0.85, 1.15))
        c = np.array([0.085 * k, 0.004 * rng.normal(), 0.004 * rng.normal()])
        bodies.append((V[F].reshape(-1, 3) + c).T.copy())
    pa = [i for i in range(len(sizes) - 1)] + [i for i in range(len(sizes) - 2)]
    pb = [i + 1 for i in range(len(sizes) - 1)] + [i + 2 for i in range(len(sizes) - 2)]
    eps_b = np.full(len(sizes), eps)
    fric = (rng.random(len(sizes)) < 0.5).astype(np.uint8)
    ids = np.arange(len(sizes)) * 10 + 3
    return bodies, pa, pb, eps_b, fric, ids


def _oracle_contacts(oracle, driver, bodies, pa, pb, eps_b, fric, ids):
    from oracle.oracle import CONTACT_DTYPE

    out = []
    hist = np.zeros(17, np.int64)
    fails = np.zeros(2, np.int64)
    for a, b in zip(pa, pb):
        c, st = oracle.detect(driver, bodies[a], bodies[a].shape[1] // 3, eps_b[a], int(fric[a]), int(ids[a]),
                              bodies[b], bodies[b].shape[1] // 3, eps_b[b], int(fric[b]), int(ids[b]), stats=True)
        out.append(c)
        hist += np.array(list(st.newton_hist))
        fails += [st.penalty_fails, st.batch_fails]
    return (np.concatenate(out) if out else np.zeros(0, CONTACT_DTYPE)), hist, fails


@pytest.mark.parametrize("driver", range(8))
def test_drivers_bit_exact_vs_oracle(ctx, oracle, driver):
    from delta_b200.detection import Meshes, detect

    for seed in (1, 2):
        bodies, pa, pb, eps_b, fric, ids = _scene(seed)
        m = Meshes.from_bodies(bodies, eps_b, fric, ids)
        out, st = detect(ctx, driver, m, pa, pb, stats=True)
        g = out.to_numpy()
        o, hist, fails = _oracle_contacts(oracle, driver, bodies, pa, pb, eps_b, fric, ids)
        assert len(g) == len(o) and len(g) > 0
        for f in FIELDS:
            assert np.array_equal(g[f], o[f], equal_nan=True), (driver, f)
        if driver == 2:
            assert list(st.newton_hist) == list(hist)
        if driver in (5, 6):
            assert [st.penalty_fails, st.batch_fails] == list(fails)


def test_bf_cert_driver_equals_bf(ctx):
    from delta_b200.detection import DRV_BF, DRV_BF_CERT, Meshes, detect

    for seed in (3, 4, 5):
        bodies, pa, pb, eps_b, fric, ids = _scene(seed, sizes=(80, 160, 40, 320, 80), eps=0.004)
        m = Meshes.from_bodies(bodies, eps_b, fric, ids)
        a = detect(ctx, DRV_BF, m, pa, pb)[0].to_numpy()
        b = detect(ctx, DRV_BF_CERT, m, pa, pb)[0].to_numpy()
        assert len(a) == len(b) and len(a) > 0
        for f in FIELDS:
            assert np.array_equal(a[f], b[f], equal_nan=True), f


def _sheet(n, z0, tilt, shift, rng):
    """Flat triangulated n x n quad grid (2*n*n triangles) over [0, 0.1]^2 at height z0,
    tilted by `tilt` about x, vertices jittered slightly."""
    g = np.linspace(0.0, 0.1, n + 1)
    X, Y = np.meshgrid(g + shift, g + shift, indexing="ij")
    Z = z0 + np.tan(tilt) * Y + 1e-5 * rng.random(X.shape)
    tris = []
    for i in range(n):
        for j in range(n):
            v00, v10 = (X[i, j], Y[i, j], Z[i, j]), (X[i + 1, j], Y[i + 1, j], Z[i + 1, j])
            v01, v11 = (X[i, j + 1], Y[i, j + 1], Z[i, j + 1]), (X[i + 1, j + 1], Y[i + 1, j + 1], Z[i + 1, j + 1])
            tris += [v00, v10, v11, v00, v11, v01]
    return np.array(tris).T.copy()


def test_bf_cert_driver_many_close_triangles(ctx, oracle):
    """Two nearly parallel sheets of 288 triangles within the contact margin of each other
    (and a sphere touching one): the certified driver's culling stages more than one
    shared-memory window of triangles per side and must still give bf's contacts."""
    from delta_b200.detection import DRV_BF, DRV_BF_CERT, Meshes, detect
    from delta_b200.scenarios import sphere_mesh

    rng = np.random.default_rng(7)
    V, F = sphere_mesh(80, rng, 0.02, (0.9, 1.1))
    sphere = (V[F].reshape(-1, 3) + np.array([0.05, 0.05, 0.0235])).T.copy()
    bodies = [_sheet(12, 0.0, 0.0, 0.0, rng), _sheet(12, 0.0015, 0.01, 0.003, rng), sphere]
    pa, pb = [0, 1, 2], [1, 2, 0]
    eps_b = np.array([0.002, 0.002, 0.002])
    fric = np.array([1, 0, 1], np.uint8)
    ids = np.array([4, 9, 11])
    m = Meshes.from_bodies(bodies, eps_b, fric, ids)
    a = detect(ctx, DRV_BF, m, pa, pb)[0].to_numpy()
    b = detect(ctx, DRV_BF_CERT, m, pa, pb)[0].to_numpy()
    o, _, _ = _oracle_contacts(oracle, DRV_BF, bodies, pa, pb, eps_b, fric, ids)
    assert len(a) > 500 and len(b) == len(a) == len(o)
    for f in FIELDS:
        assert np.array_equal(a[f], b[f], equal_nan=True), f
        assert np.array_equal(b[f], o[f], equal_nan=True), f


def test_golden_driver_fixture(ctx, golden):
    from delta_b200 import detection

    g = golden["drivers"]
    A, B, nA, nB, eps = g["A"], g["B"], int(g["nA"]), int(g["nB"]), float(g["eps"])
    fns = [detection.bf, detection.penalty, detection.penaltyStat, detection.hybridWithPerBatchFallBack,
           detection.hybridWithPerTriangleFallBack, detection.hybridBatchStat, detection.hybridTriangleStat]
    for d, fn in enumerate(fns):
        c = fn(A[0], A[1], A[2], nA, eps, True, 3, B[0], B[1], B[2], nB, eps, True, 8, ctx=ctx)
        ref = g[f"contacts_{d}"]
        assert len(c) == len(ref)
        for f in FIELDS[:10]:
            assert np.array_equal(c[f], ref[f], equal_nan=True), (d, f)


def test_capacity_error_reports_needed_size(ctx):
    from delta_b200._lib import DeltaError
    from delta_b200.detection import Meshes, detect

    bodies, pa, pb, eps_b, fric, ids = _scene(1)
    m = Meshes.from_bodies(bodies, eps_b, fric, ids)
    full = detect(ctx, 0, m, pa, pb)[0]
    assert full.count > 2
    with pytest.raises(DeltaError, match="CAPACITY"):
        detect(ctx, 0, m, pa, pb, capacity=2, grow=False)
    again = detect(ctx, 0, m, pa, pb, capacity=2, grow=True)[0]
    assert again.count == full.count


def test_bad_body_index_is_rejected(ctx):
    from delta_b200._lib import DeltaError
    from delta_b200.detection import Meshes, detect

    bodies, pa, pb, eps_b, fric, ids = _scene(1)
    m = Meshes.from_bodies(bodies, eps_b, fric, ids)
    with pytest.raises(DeltaError, match="INVALID"):
        detect(ctx, 0, m, [0], [len(bodies)])


def test_empty_pair_list(ctx):
    from delta_b200.detection import Meshes, detect

    bodies, pa, pb, eps_b, fric, ids = _scene(1)
    m = Meshes.from_bodies(bodies, eps_b, fric, ids)
    out, _ = detect(ctx, 0, m, [], [])
    assert out.count == 0
