"""The zoltan/ part of the oracle (oracle/zoltan_oracle.c) against the reference's own
zoltan/bf.cpp, penalty.cpp and hybrid.cpp compiled here (oracle/_ref/libzoltan_ref.so,
bit for bit), and property checks of its dynamics and forces, whose reference files need
the Zoltan and MPI headers and are not built here."""
import numpy as np
import pytest

from tests import zoltan_cases


@pytest.fixture(scope="module")
def zref():
    from oracle.oracle import ZoltanReference

    if not ZoltanReference.available():
        pytest.skip("oracle/_ref/libzoltan_ref.so not built (the reference sources are absent)")
    return ZoltanReference()


def _same(x, y):
    return np.array_equal(x, y, equal_nan=True)


def _list(n, seed, degenerate=True):
    from delta_b200.scenarios import narrowphase_pairs

    a, b, _, _ = narrowphase_pairs(n, seed=seed)
    if degenerate:  # zero cross products: B1 = B0, B2 = B1, a flat A
        b[3:6, :5] = b[0:3, :5]
        b[6:9, 5:10] = b[3:6, 5:10]
        a[3:6, 10:15] = a[0:3, 10:15]
    return a, b


def test_zoltan_bf_per_pair_equals_reference(oracle, zref):
    a, b = _list(1 << 13, seed=31)
    p0 = np.full((3, a.shape[1]), 7.0)
    po, qo = oracle.zoltan_bf_pairs(a, b, p0, p0)
    pr, qr = zref.zoltan_bf_pairs(a, b, p0, p0)
    assert _same(po, pr) and _same(qo, qr)
    assert np.all(po[:, :10] == 7.0)  # the early returns leave the outputs untouched


@pytest.mark.parametrize("method", ["penalty", "hybrid"])
@pytest.mark.parametrize("it,cut", [(0, 0), (1, 3), (2, 1)])
def test_zoltan_soa_equals_reference(oracle, zref, method, it, cut):
    a, b = _list(1 << 12, seed=32)
    d, e, f = b[0:3], b[3:6], b[6:9]
    n = d.shape[1]
    p0 = np.full((3, n), -3.0)
    for j in (0, 11, 400):  # the single triangle: a general one and a degenerate one
        abc = a[:, j].reshape(3, 3)
        po, qo = oracle.zoltan_soa(method, it, n - cut, abc, d, e, f, p0, p0)
        pr, qr = zref.zoltan_soa(method, it, n - cut, abc, d, e, f, p0, p0)
        assert _same(po, pr) and _same(qo, qr), (method, j)


def test_zoltan_hybrid_falls_back_in_some_batches(oracle):
    a, b = _list(1 << 12, seed=33, degenerate=False)
    p, q = oracle.zoltan_soa("hybrid", 0, b.shape[1], a[:, 0].reshape(3, 3), b[0:3], b[3:6], b[6:9])
    P = p.reshape(3, -1, 4)
    fell_back = np.all(P == P[:, :, :1], axis=(0, 2))
    assert 0.05 < fell_back.mean() < 0.95


def test_zoltan_bf_soa_is_the_per_pair_loop(oracle, zref):
    a, b = _list(2000, seed=34)
    abc = a[:, 3].reshape(3, 3)
    n = b.shape[1]
    p0 = np.full((3, n), 5.0)
    p, q = oracle.zoltan_soa("bf_soa", 7, n - 2, abc, b[0:3], b[3:6], b[6:9], p0, p0)
    A = np.repeat(abc.reshape(9, 1), n, 1)
    pr, qr = zref.zoltan_bf_pairs(A, b, p0, p0)
    assert _same(p[:, 7:n - 2], pr[:, 7:n - 2]) and _same(q[:, 7:n - 2], qr[:, 7:n - 2])
    assert np.all(p[:, :7] == 5.0) and np.all(p[:, n - 2:] == 5.0)


def test_zoltan_force_balances_in_pairs(oracle):
    """Contact forces act equal and opposite on master and slave at the same point: the
    total force is the total weight, and the total torque about the origin equals the
    weight's moment (up to rounding)."""
    s = zoltan_cases.system(nb=48, seed=3)
    c = zoltan_cases.contacts(nb=48, seed=3)
    g = np.array([0.0, -9.81, 0.0])
    nb = 48
    F0 = np.zeros((3, nb)); T0 = np.zeros((3, nb))
    F, T = oracle.zoltan_force(c["offset"], c["slave"], c["point"], c["normal"], c["depth"], s["position"],
                               s["angular"], s["linear"], s["mass"], F0, T0, g, 1e2, 1.0)
    W = s["mass"][None] * g[:, None]
    assert np.allclose(F.sum(1), W.sum(1), rtol=0, atol=1e-10 * np.abs(F).sum())
    x = s["position"][:3]
    L = np.cross(x.T, F.T).sum(0) + T.sum(1)
    Lw = np.cross(x.T, W.T).sum(0)
    assert np.allclose(L, Lw, rtol=0, atol=1e-10 * (np.abs(T).sum() + np.abs(np.cross(x.T, F.T)).sum()))


def test_zoltan_update_matches_delta_dynamics_up_to_association(oracle):
    """zoltan's update is delta's updateAngular + updateRotationMatrix + the move, with
    the sums of NVADDMUL associated differently: the two agree to rounding."""
    s = zoltan_cases.system(nb=16, seed=4, omega=0.5)
    dt = 1e-3
    t, ang, lin, rot, pos, F, T = oracle.zoltan_update(s["t"], s["pid"], s["angular"], s["linear"], s["rotation"],
                                                       s["position"], s["inertia"], s["inverse"], s["mass"],
                                                       s["force"], s["torque"], dt)
    assert np.all(F == 0) and np.all(T == 0)
    for i in range(16):
        W = s["angular"][:3, i].copy()
        R = s["rotation"][:, i].copy()
        J, Ji, tq = (np.ascontiguousarray(s[k][:, i]) for k in ("inertia", "inverse", "torque"))
        oracle.lib.dor_update_angular(W.ctypes.data, R.ctypes.data, J.ctypes.data, Ji.ctypes.data, tq.ctypes.data, dt)
        w = np.zeros(3)
        oracle.lib.dor_update_rotation(w.ctypes.data, W.ctypes.data, R.ctypes.data, dt)
        assert np.allclose(ang[:3, i], W, rtol=1e-13, atol=1e-15)
        assert np.allclose(rot[:, i], R, rtol=1e-13, atol=1e-15)
        assert np.allclose(ang[3:, i], w, rtol=1e-13, atol=1e-15)
        v = s["linear"][:, i] + dt / s["mass"][i] * s["force"][:, i]
        assert np.allclose(lin[:, i], v, rtol=1e-14) and np.allclose(pos[:3, i], s["position"][:3, i] + dt * v)
    # the spatial vertices follow their bodies: x + L (X_ref - X_centre)
    R = rot[:, s["pid"]].reshape(3, 3, -1)  # [col][row]
    for v in range(3):
        C = s["t"][3 + v] - pos[3:6, s["pid"]]
        x = pos[:3, s["pid"]] + np.einsum("crn,cn->rn", R, C)
        assert np.allclose(t[v], x, rtol=0, atol=1e-14)
    assert np.array_equal(t[3:], s["t"][3:])


def test_zoltan_integrate_reflects_at_the_box(oracle):
    rng = np.random.default_rng(9)
    nt = 500
    t = rng.uniform(-1.05, 1.05, (3, 3, nt))
    v = rng.normal(size=(3, nt))
    t2, v2 = oracle.zoltan_integrate(0.01, [-1, -1, -1], [1, 1, 1], t, v)
    assert np.array_equal(t2, t + 0.01 * v[None])
    flips = sum(((t2[w] < -1) | (t2[w] > 1)).astype(int) for w in range(3))
    assert np.array_equal(v2, np.where(flips % 2 == 1, -v, v))
