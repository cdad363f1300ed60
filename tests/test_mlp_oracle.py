"""The learned warm start's CPU oracle (no GPU): its calculus, its rounding and its
features, checked before it is used to check the CUDA kernels."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo


def _params(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    d = {}
    for l, (fi, fo) in enumerate(mo.LAYERS, start=1):
        d[f"W{l}"] = rng.normal(0, scale / np.sqrt(fi), (fo, fi))
        d[f"b{l}"] = rng.normal(0, 0.1, fo)
    return d


def test_layout_matches_architecture():
    L = mo.layout()
    assert L["W1"] == 0 and L["b1"] == 128 * 32 and L["W2"] == L["b1"] + 128
    assert L["b4"] == L["W4"] + 4 * 128 and L["total"] % 8 == 0 and L["total"] >= L["b4"] + 4
    d = _params()
    back = mo.unpack(mo.pack(d))
    for k in d:
        assert np.array_equal(back[k], d[k])


def test_bf16_rounding_is_round_to_nearest_even():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(0, 10, 20000), rng.normal(0, 1e-3, 20000), [0.0, -0.0, 1.0, 3.0, 1 + 2 ** -8]])
    x = x.astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(mo.bf16(x), ref)


def test_gradients_match_finite_differences():
    """FP64 (unrounded) backward against central differences of the FP64 loss."""
    rng = np.random.default_rng(1)
    M = 64
    X = np.zeros((M, 32))
    X[:, :18] = rng.normal(0, 0.5, (M, 18))
    T = rng.uniform(0, 1, (M, 4))
    valid = rng.uniform(size=M) > 0.1
    P = _params(2)
    cache = mo.forward(X, P, rounded=False)
    loss, g = mo.backward(cache, P, T, valid, rounded=False)

    def f(Pm):
        return mo.backward(mo.forward(X, Pm, rounded=False), Pm, T, valid, rounded=False)[0]

    h = 1e-6
    for name in ("W1", "b1", "W2", "b3", "W4", "b4"):
        idx = [tuple(rng.integers(0, s) for s in P[name].shape) for _ in range(6)]
        for ix in idx:
            Pp = {k: v.copy() for k, v in P.items()}
            Pm = {k: v.copy() for k, v in P.items()}
            Pp[name][ix] += h
            Pm[name][ix] -= h
            fd = (f(Pp) - f(Pm)) / (2 * h)
            assert abs(fd - g[name][ix]) <= 1e-6 * max(1.0, abs(fd)), (name, ix, fd, g[name][ix])


def test_gelu_grad_matches_difference():
    x = np.linspace(-6, 6, 1001)
    h = 1e-6
    fd = (mo.gelu(x + h) - mo.gelu(x - h)) / (2 * h)
    assert np.max(np.abs(fd - mo.gelu_grad(x))) < 1e-8


def test_canon_features_invariant_and_targets_reconstruct():
    """Features do not change under a rigid motion + uniform scaling of the pair (beyond
    rounding), and the targets reconstruct the closest points."""
    from delta_b200.scenarios import narrowphase_pairs

    from oracle.oracle import Oracle

    a, b, _, _ = narrowphase_pairs(512, seed=5, intersecting=0.0)
    p, q, _, _ = Oracle().pairs(0, a, b)
    f, T, ok = mo.canon(a, b, p, q)
    assert ok.mean() > 0.99
    rng = np.random.default_rng(0)
    Qm, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    shift, sc = rng.normal(size=3), 2.5
    move = lambda x: (sc * (Qm @ x.reshape(3, 3, -1).transpose(1, 0, 2).reshape(3, -1)).reshape(3, 3, -1)  # noqa: E731
                      .transpose(1, 0, 2).reshape(9, -1) + np.tile(shift, 3)[:, None])
    f2, _, _ = mo.canon(move(a), move(b))
    assert np.max(np.abs(f2 - f)[ok]) < 2e-2  # a BF16 step at most
    for tri, pts, k in ((a, p, 0), (b, q, 2)):
        V = [tri[3 * v:3 * v + 3] for v in range(3)]
        rec = V[0] + T[:, k] * (V[1] - V[0]) + T[:, k + 1] * (V[2] - V[0])
        err = np.abs(rec - pts).max(0)
        assert np.all(err[ok] < 1e-5)
