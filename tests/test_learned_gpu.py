"""The learned warm start on the GPU: its kernels against the CPU oracle
(oracle/mlp_oracle.py) and torch's FP32 matmul, training with the library's own
forward/backward kernels, what the trained network gains over the same solver without
it, and the learned solver's results against FP64 bfSolver.

Tolerances: BF16 tensor-core GEMM vs torch FP32 matmul of the same BF16 operands:
relative Frobenius error <= 1e-5.  Forward/backward vs the oracle with the BF16
roundings mirrored: relative Frobenius error <= 2e-2 per tensor (what remains is FP32
versus FP64 accumulation and rare one-step BF16 rounding flips that follow from it),
no element off by more than 5% of the tensor's largest entry and the median element
within 1%.  The GPU backward also matches central differences of the GPU loss along a
random direction per tensor within 5%.
Learned solver vs FP64 bfSolver: relative distance error <= 1e-6 on every pair.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _rel(x, y):
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-30))


@pytest.fixture(scope="module")
def pairs():
    from delta_b200.scenarios import narrowphase_pairs

    a, b, _, _ = narrowphase_pairs(1 << 16, seed=77)
    return a, b


def test_layout_matches_oracle():
    from delta_b200.learned import layout

    from oracle import mlp_oracle as mo

    assert layout() == mo.layout()


@pytest.mark.parametrize("engine", ["tcgen05", "mma"])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("split,acc", [(1, 0), (4, 0), (1, 1), (3, 1)])
@pytest.mark.parametrize("shape", [(200, 72, 300), (130, 4, 37), (4, 128, 1000), (300, 136, 4)])
def test_gemm_bf16_vs_torch(ctx, engine, ta, tb, split, acc, shape):
    """The training GEMM on both engines against torch's FP32 matmul of the same BF16
    operands, for the shapes training uses (N or M of 4: the output layer; K of 4: its
    backward) and ragged ones."""
    import torch

    from delta_b200._lib import check, lib
    from delta_b200.learned import set_engine

    set_engine(ctx, engine)
    g = torch.Generator(device="cuda").manual_seed(ta * 7 + tb * 3 + split)
    M, N, K = shape
    A = torch.randn((K, M) if ta else (M, K), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((N, K) if tb else (K, N), generator=g, device="cuda").to(torch.bfloat16)
    C0 = torch.randn((M, N), generator=g, device="cuda")
    Cm = C0.clone()
    check(lib().delta_gemm_bf16(ctx.handle, M, N, K, A.data_ptr(), A.shape[1], ta, B.data_ptr(), B.shape[1], tb,
                                Cm.data_ptr(), N, acc, split))
    ctx.synchronize()
    ctx.synchronize()
    set_engine(ctx, "tcgen05")
    Af = A.float().T if ta else A.float()
    Bf = B.float().T if tb else B.float()
    ref = Af @ Bf + (C0 if acc else 0)
    assert _rel(Cm.cpu(), ref.cpu()) <= 1e-5


@pytest.mark.parametrize("split", [1, 32])
def test_gemm_bf16_weight_gradient_shape(ctx, split):
    """A weight-gradient GEMM as training runs it (dW = d^T prev: both operands transposed,
    K = the batch, split-K, accumulate) on the tcgen05 engine against torch."""
    import torch

    from delta_b200._lib import check, lib
    from delta_b200.learned import set_engine

    set_engine(ctx, "tcgen05")
    g = torch.Generator(device="cuda").manual_seed(split)
    M, N, K = 128, 128, 16384
    A = torch.randn((K, M), generator=g, device="cuda").to(torch.bfloat16)
    B = torch.randn((K, N), generator=g, device="cuda").to(torch.bfloat16)
    C0 = torch.randn((M, N), generator=g, device="cuda")
    Cm = C0.clone()
    check(lib().delta_gemm_bf16(ctx.handle, M, N, K, A.data_ptr(), M, 1, B.data_ptr(), N, 0, Cm.data_ptr(), N, 1,
                                split))
    ctx.synchronize()
    # FP64 reference: with K = 16384 one FP32 accumulation chain (split 1) carries a relative
    # rounding error of order sqrt(K) * 2^-24 ~ 1e-5, as torch's own FP32 matmul does
    ref = A.double().T @ B.double() + C0.double()
    assert _rel(Cm.cpu(), ref.cpu()) <= 4e-5


def test_features_bit_exact_vs_oracle(ctx, pairs):
    from delta_b200.learned import features
    from delta_b200.narrowphase import pairs_device

    from oracle import mlp_oracle as mo

    a, b = pairs
    da, db = _dev(a), _dev(b)
    p, q, _, _ = pairs_device(ctx, 0, da, db)
    X, T, valid = features(ctx, da, db, p, q)
    ctx.synchronize()
    f, To, ok = mo.canon(a, b, p.cpu().numpy(), q.cpu().numpy())
    assert np.array_equal(X.float().cpu().numpy().astype(np.float64), f)
    assert np.array_equal(valid.cpu().numpy().astype(bool), ok)
    assert np.array_equal(T.cpu().numpy(), To)


def test_forward_backward_vs_oracle(ctx, pairs):
    import torch

    from delta_b200.learned import WarmStartMLP, labelled

    from oracle import mlp_oracle as mo

    a, b = pairs
    M = 4096
    da, db = _dev(a[:, :M]), _dev(b[:, :M])
    X, T, valid = labelled(ctx, da, db)
    model = WarmStartMLP(ctx, seed=3)
    nv = int(valid.sum().item())
    Y = model.forward(X).clone()
    model.backward(X, T, valid, nv)
    ctx.synchronize()
    P = mo.unpack(model.params.cpu().numpy().astype(np.float64))
    cache = mo.forward(X.float().cpu().numpy(), P)
    loss, g = mo.backward(cache, P, T.cpu().numpy().astype(np.float64), valid.cpu().numpy().astype(bool))
    assert _rel(Y.cpu().numpy(), cache["Y"]) <= 2e-2
    assert abs(float(model.loss.item()) - loss) <= 2e-2 * loss
    for name in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        gg = model.grad(name).cpu().numpy().astype(np.float64)
        assert _rel(gg, g[name]) <= 2e-2, name
        # per element: no entry off by more than 5% of the tensor's largest gradient, and
        # the typical entry within 1% of its own value
        err = np.abs(gg - g[name])
        assert err.max() <= 5e-2 * np.abs(g[name]).max(), name
        big = np.abs(g[name]) > 1e-3 * np.abs(g[name]).max()
        assert np.median(err[big] / np.abs(g[name][big])) <= 1e-2, name
    # and the Adam step against the oracle's
    w0 = model.params.cpu().numpy().astype(np.float64)
    gr = model.grads.cpu().numpy().astype(np.float64)
    model.adam(lr=1e-3)
    ctx.synchronize()
    w1, _, _ = mo.adam(w0, gr, np.zeros_like(w0), np.zeros_like(w0), 1)
    assert np.max(np.abs(model.params.cpu().numpy() - w1)) <= 1e-6
    assert torch.equal(model.params_bf16, model.params.to(torch.bfloat16))


def test_backward_matches_directional_finite_differences(ctx, pairs):
    """The GPU backward against central differences of the GPU forward + MSE loss, per
    tensor, along the sign pattern of the tensor's GPU gradient scaled to 5% of the
    tensor's RMS (a wrong gradient -- a transposed block, a wrong sign -- predicts the
    change of a direction it did not choose).  The applied perturbation is the one the
    forward sees (weights are used as BF16, biases as FP32), and <g, dW> must predict
    L(W+) - L(W-) within 5%."""
    import torch

    from delta_b200.learned import WarmStartMLP, labelled

    a, b = pairs
    M = 4096
    X, T, valid = labelled(ctx, _dev(a[:, :M]), _dev(b[:, :M]))
    nv = int(valid.sum().item())
    model = WarmStartMLP(ctx, seed=11)
    L = model.L

    def loss_at(params):
        model.params.copy_(params)
        model._refresh_bf16()
        model.forward(X)
        model.backward(X, T, valid, nv)
        ctx.synchronize()
        return float(model.loss.item()), model.params_bf16.double().clone()

    p0 = model.params.clone()
    loss_at(p0)
    g = model.grads.double().clone()
    for name in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        o = L[name]
        size = model.grad(name).numel()
        v = torch.sign(g[o:o + size]).float()
        step = 5e-2 * float(p0[o:o + size].pow(2).mean().sqrt())
        pp, pm = p0.clone(), p0.clone()
        pp[o:o + size] += step * v
        pm[o:o + size] -= step * v
        lp, bp = loss_at(pp)
        lm, bm = loss_at(pm)
        if name[0] == "W":
            dw = (bp - bm)[o:o + size]
        else:
            dw = (pp.double() - pm.double())[o:o + size]
        pred = float((g[o:o + size] * dw).sum())
        assert abs((lp - lm) - pred) <= 5e-2 * abs(pred) + 1e-9, (name, lp - lm, pred)
    model.params.copy_(p0)
    model._refresh_bf16()


def test_fused_inference_equals_layer_path(ctx, pairs):
    from delta_b200.learned import WarmStartMLP, features

    a, b = pairs
    n = 5000  # not a multiple of the 16-row tile
    da, db = _dev(a[:, :n]), _dev(b[:, :n])
    model = WarmStartMLP(ctx, seed=4)
    x0 = model.predict(da, db)
    X, _, _ = features(ctx, da, db)
    Y = model.forward(X)
    ctx.synchronize()
    assert np.array_equal(x0.cpu().numpy(), Y.cpu().numpy())


def test_tcgen05_inference_matches_mma_path_and_oracle(ctx, pairs):
    """The tcgen05/TMEM inference kernel against the mma.sync kernel (same network, other
    accumulation order: equal to BF16 rounding) and against the oracle's forward."""
    from delta_b200.learned import WarmStartMLP, features

    from oracle import mlp_oracle as mo

    a, b = pairs
    n = 40000  # several 128-pair tiles per CTA, last tile partial
    da, db = _dev(a[:, :n]), _dev(b[:, :n])
    model = WarmStartMLP.load(ctx)
    x_mma = model.predict(da, db).cpu().numpy()
    x_tc = model.predict(da, db, engine="tcgen05").cpu().numpy()
    assert np.all(np.isfinite(x_tc))
    assert _rel(x_tc, x_mma) <= 1e-2
    assert np.max(np.abs(x_tc - x_mma)) <= 5e-2
    X, _, _ = features(ctx, da[:, :4096].contiguous(), db[:, :4096].contiguous())
    P = mo.unpack(model.params.cpu().numpy().astype(np.float64))
    ref = mo.forward(X.float().cpu().numpy(), P)["Y"]
    assert _rel(x_tc[:4096], ref) <= 2e-2


@pytest.fixture(scope="module")
def trained(ctx):
    """A network trained on 2^19 fresh pairs for 6 epochs with the library's kernels."""
    from delta_b200.learned import WarmStartMLP, labelled, train
    from delta_b200.scenarios import narrowphase_pairs

    a, b, _, _ = narrowphase_pairs(1 << 19, seed=2024)
    X, T, valid = labelled(ctx, _dev(a), _dev(b))
    model = WarmStartMLP(ctx, seed=0)
    losses = train(model, X, T, valid, epochs=6, batch=8192, lr=2e-3, seed=1)
    return model, losses


def test_training_reduces_loss(trained):
    _, losses = trained
    assert losses[-1] < 0.5 * losses[0], losses
    assert all(np.isfinite(losses))


def test_trained_network_beats_centroid_start(ctx, trained, pairs):
    """What the network gains: the reference penalty iteration (penalty.cpp:434-582)
    converges in fewer iterations from the prediction than from 0.33, and the learned
    solver certifies more pairs without the fallback than from the centroids."""
    import torch

    from delta_b200._lib import check, lib
    from delta_b200.learned import refine

    model, _ = trained
    a, b = pairs
    da, db = _dev(a), _dev(b)
    n = a.shape[1]
    x0 = model.predict(da, db)
    it = {}
    for name, start in (("net", x0), ("plain", None)):
        p = torch.empty((3, n), dtype=torch.float64, device="cuda")
        q, d = torch.empty_like(p), torch.empty(n, dtype=torch.float64, device="cuda")
        iters = torch.empty(n, dtype=torch.uint8, device="cuda")
        check(lib().delta_penalty_warm(ctx.handle, n, da.data_ptr(), db.data_ptr(), n,
                                       None if start is None else start.data_ptr(), 1e-6, p.data_ptr(),
                                       q.data_ptr(), d.data_ptr(), iters.data_ptr()))
        it[name] = iters.float().mean().item()
    assert it["net"] < it["plain"], it
    for sweeps in (0, 1):
        c_net = refine(ctx, da, db, x0, sweeps)[3].float().mean().item()
        c_plain = refine(ctx, da, db, None, sweeps)[3].float().mean().item()
        assert c_net > c_plain, (sweeps, c_net, c_plain)


@pytest.mark.parametrize("features", [3, 7, 11, 15])
@pytest.mark.parametrize("use_net", [True, False])
def test_learned_solver_vs_fp64_bf(ctx, trained, oracle, pairs, use_net, features):
    """Every pair within 1e-6 relative distance of FP64 bfSolver; uncertified pairs
    (fallback) bit-exact; contact sets equal outside the 1e-6 band of the threshold."""
    from delta_b200.learned import learned_pairs

    from tests.golden.make_golden import edge_case_pairs

    model = trained[0] if use_net else None
    ea, eb = edge_case_pairs()
    a = np.concatenate([pairs[0], ea], 1)
    b = np.concatenate([pairs[1], eb], 1)
    p, q, d, flags, nfb = learned_pairs(ctx, model, _dev(a), _dev(b), sweeps=2, count_fallback=True,
                                        features=features)
    ctx.synchronize()
    p, q, d, flags = p.cpu().numpy(), q.cpu().numpy(), d.cpu().numpy(), flags.cpu().numpy()
    assert set(np.unique(flags)) <= {1, 2} and nfb == int((flags == 2).sum())
    op, oq, od, _ = oracle.pairs(0, a, b)
    fin = np.isfinite(od)
    rel = np.abs(d - od)[fin] / np.maximum(od[fin], 1e-300)
    assert rel.max() <= 1e-6, rel.max()
    fb = flags == 2
    assert np.array_equal(d[fb], od[fb], equal_nan=True)
    assert np.array_equal(p[:, fb], op[:, fb], equal_nan=True)
    assert np.array_equal(q[:, fb], oq[:, fb], equal_nan=True)
    assert (flags == 1).mean() > 0.5
    for thr in (1e-4, 1e-3, 1e-2):
        band = np.abs(od - thr) <= 1e-6 * thr
        assert np.array_equal((d <= thr)[~band], (od <= thr)[~band])


@pytest.mark.parametrize("engine", ["tcgen05", "mma"])
def test_learned_pipeline_engines(ctx, oracle, pairs, engine):
    """The bundled network on either tensor-core engine inside delta_pairs_run_learned:
    within 1e-6 of FP64 bfSolver, fallback bit-exact, no time-out."""
    from delta_b200.learned import WarmStartMLP, learned_pairs, set_engine

    a, b = pairs[0][:, :30000], pairs[1][:, :30000]
    model = WarmStartMLP.load(ctx)
    set_engine(ctx, engine)
    try:
        p, q, d, fl, nf = learned_pairs(ctx, model, _dev(a), _dev(b), sweeps=0, count_fallback=True)
    finally:
        set_engine(ctx, "tcgen05")
    d, fl = d.cpu().numpy(), fl.cpu().numpy()
    _, _, od, _ = oracle.pairs(0, a, b)
    fin = np.isfinite(od)
    assert np.all(np.abs(d - od)[fin] <= 1e-6 * od[fin])
    assert np.array_equal(d[fl == 2], od[fl == 2], equal_nan=True)
    assert (fl == 1).mean() > 0.8  # the trained network's start certifies most pairs without sweeps


def test_learned_host_entry_equals_device_entry(ctx, trained, pairs):
    """delta_pairs_run_learned_host gives the device entry point's results bit for bit."""
    from delta_b200.learned import learned_pairs, learned_pairs_host

    a, b = pairs[0][:, :20000], pairs[1][:, :20000]
    model = trained[0]
    p, q, d, fl, nf = learned_pairs(ctx, model, _dev(a), _dev(b), sweeps=1, count_fallback=True, features=7)
    hp, hq, hd, hfl, hnf = learned_pairs_host(ctx, model, a, b, sweeps=1, features=7)
    assert nf == hnf
    assert np.array_equal(p.cpu().numpy(), hp) and np.array_equal(q.cpu().numpy(), hq)
    assert np.array_equal(d.cpu().numpy(), hd) and np.array_equal(fl.cpu().numpy(), hfl)


def test_learned_rejects_bad_arguments(ctx, pairs):
    from delta_b200._lib import DeltaError
    from delta_b200.learned import learned_pairs

    a, b = _dev(pairs[0][:, :100]), _dev(pairs[1][:, :100])
    with pytest.raises(DeltaError):
        learned_pairs(ctx, None, a, b, sweeps=1, features=5)
    with pytest.raises(DeltaError):
        learned_pairs(ctx, None, a, b, sweeps=-1)


def test_learned_host_pipeline_many_chunks(ctx, trained):
    """The pipelined host entry (several chunks, pitched host arrays) equals the device entry."""
    from delta_b200.learned import learned_pairs, learned_pairs_host
    from delta_b200.scenarios import narrowphase_pairs

    n = (1 << 20) + 12345
    a, b, _, _ = narrowphase_pairs(n, seed=31)
    model = trained[0]
    p, q, d, fl, nf = learned_pairs(ctx, model, _dev(a), _dev(b), sweeps=1, count_fallback=True, features=3)
    hp, hq, hd, hfl, hnf = learned_pairs_host(ctx, model, a, b, sweeps=1, features=3)
    assert nf == hnf > 0
    assert np.array_equal(d.cpu().numpy(), hd) and np.array_equal(fl.cpu().numpy(), hfl)
    assert np.array_equal(p.cpu().numpy(), hp) and np.array_equal(q.cpu().numpy(), hq)


@pytest.mark.parametrize("shift,scale", [(1e4, 1.0), (-3e2, 1.0), (0.0, 1e-5), (5.0, 1e3)])
def test_learned_solver_translated_and_scaled(ctx, oracle, pairs, shift, scale):
    """Pairs moved far from the origin or scaled: the certificate's rounding slack grows
    with the coordinates, so pairs it cannot certify go to the exact solver; every result
    stays within 1e-6 of FP64 bfSolver on the same (moved) inputs, fallback bit-exact."""
    from delta_b200.learned import learned_pairs

    a = pairs[0][:, :20000] * scale + shift
    b = pairs[1][:, :20000] * scale + shift
    p, q, d, fl, nf = learned_pairs(ctx, None, _dev(a), _dev(b), sweeps=2, count_fallback=True, features=3)
    d, fl = d.cpu().numpy(), fl.cpu().numpy()
    _, _, od, _ = oracle.pairs(0, a, b)
    fin = np.isfinite(od)
    assert np.all(np.abs(d - od)[fin] <= 1e-6 * od[fin])
    assert np.array_equal(d[fl == 2], od[fl == 2], equal_nan=True)
    assert nf == int((fl == 2).sum())


def test_tcgen05_bounded_wait_reports_timeout_and_context_stays_usable(ctx, pairs):
    """The tcgen05 kernel's wait for the tensor cores is bounded: with the first layer's
    commit withheld (nothing arrives on the barrier, nothing is in flight) the wait runs
    out, the kernel frees its TMEM and the call reports DELTA_ERR_TIMEOUT.  The same
    context then runs the network normally."""
    import torch

    from delta_b200._lib import DeltaError, check, lib
    from delta_b200.learned import WarmStartMLP

    a, b = pairs[0][:, :1000], pairs[1][:, :1000]
    da, db = _dev(a), _dev(b)
    model = WarmStartMLP.load(ctx)
    x0 = torch.empty((1000, 4), dtype=torch.float32, device="cuda")
    for _ in range(2):
        with pytest.raises(DeltaError, match="TIMEOUT"):
            check(lib().delta_mlp_infer_tcgen05_wait_test(ctx.handle, 1000, da.data_ptr(), db.data_ptr(), 1000,
                                                          model.params.data_ptr(), model.params_bf16.data_ptr(),
                                                          x0.data_ptr(), 1 << 14))
    x_tc = model.predict(da, db, engine="tcgen05").cpu().numpy()
    x_mma = model.predict(da, db).cpu().numpy()
    assert _rel(x_tc, x_mma) <= 1e-2
