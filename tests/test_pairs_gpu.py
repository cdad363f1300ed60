"""Pair-list kernels (libdelta_b200.so on the GPU) against the oracle.

FP64 methods reproduce the reference arithmetic and must match bit for bit.  BF_CERT
(FP32 filter, FP64 finish) must equal FP64 bf bit for bit.  FP32 methods are checked
against FP64 with the tolerances written in each test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

METHODS = {"bf": 0, "penalty": 1, "penalty_iter": 2, "gjk": 3, "hybrid": 4}
MAX_ERR = 1e-3


@pytest.fixture(scope="module")
def workload():
    from delta_b200.scenarios import narrowphase_pairs
    from tests.golden.make_golden import edge_case_pairs

    a, b, d, cls = narrowphase_pairs(1 << 16, seed=1234)
    ea, eb = edge_case_pairs()
    return np.concatenate([a, ea], 1), np.concatenate([b, eb], 1)


def _differ(x, y):
    """Columns where x and y differ bit for bit (NaN equals NaN)."""
    return ~((x == y) | (np.isnan(x) & np.isnan(y))).all(0)


def _dev(x):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _run(ctx, method, a, b, precision=0):
    from delta_b200.narrowphase import pairs_device

    p, q, d, fl = pairs_device(ctx, method, _dev(a), _dev(b), precision=precision, max_error=MAX_ERR)
    ctx.synchronize()
    return p.cpu().numpy(), q.cpu().numpy(), d.cpu().numpy(), fl.cpu().numpy()


@pytest.mark.parametrize("name", list(METHODS))
def test_f64_methods_bit_exact_vs_oracle(ctx, oracle, workload, name):
    a, b = workload
    m = METHODS[name]
    gp, gq, gd, gf = _run(ctx, m, a, b)
    op, oq, od, of = oracle.pairs(m, a, b, max_error=MAX_ERR)
    bad = np.flatnonzero(_differ(gp, op) | _differ(gq, oq) | _differ(gd[None], od[None]))
    assert bad.size == 0, f"{bad.size} pairs differ, first {bad[:5]}"
    assert np.array_equal(gf, of)


@pytest.mark.parametrize("name", list(METHODS))
def test_f64_methods_match_golden(ctx, golden, name):
    g = golden["pairs"]
    gp, gq, gd, gf = _run(ctx, METHODS[name], g["a"], g["b"])
    assert np.array_equal(gp, g[f"{name}_p"], equal_nan=True) and np.array_equal(gq, g[f"{name}_q"], equal_nan=True)
    assert np.array_equal(gd, g[f"{name}_d"], equal_nan=True) and np.array_equal(gf, g[f"{name}_flags"])


def test_bf_cert_equals_f64_bf(ctx, oracle, workload):
    a, b = workload
    gp, gq, gd, ev = _run(ctx, 5, a, b)
    op, oq, od, _ = oracle.pairs(0, a, b)
    bad = np.flatnonzero(_differ(gp, op) | _differ(gq, oq) | _differ(gd[None], od[None]))
    assert bad.size == 0, f"{bad.size} pairs differ, first {bad[:5]}"
    assert ev.min() >= 1 and ev.max() <= 15


def test_f32_bf_close_to_f64(ctx, oracle, workload):
    """FP32 bfSolver (the reference's iREAL=float build) against FP64: the algorithm is
    poorly conditioned in FP32 for some pairs, so the bound is statistical:
    |d32 - d64| <= 1e-5 * (1 + d64) on at least 99.5% of pairs, and <= 1e-3 on all."""
    a, b = workload
    _, _, d32, _ = _run(ctx, 0, a, b, precision=1)
    _, _, d64, _ = oracle.pairs(0, a, b)
    err = np.abs(d32 - d64)
    assert np.all(np.isfinite(d32))
    assert np.mean(err <= 1e-5 * (1 + d64)) >= 0.995
    assert err.max() <= 1e-3


# Error of each FP32 method (the reference's iREAL=float algorithm) against the same method
# in FP64 (the oracle, which equals the reference's FP64 build bit for bit), per class of
# the narrowphase microbenchmark draw.  rel = |d32 - d64| / d64 over pairs with d64 > 0;
# abs = |d32 - d64| (the triangles span ~1).  The bounds are the values measured on 2^20
# pairs of the same distribution with a margin of about 3x; they state how far the plain
# FP32 methods are from FP64 (small separations are poorly conditioned in FP32, and the
# FP32 GJK stops early on about 1% of pairs).  The certified FP32 paths (BF_CERT, the
# learned hybrid) are the ones held to 1e-6.  None: not bounded (relative error of
# intersecting pairs, whose FP64 distance is near 0).
F32_BOUNDS = {  # method: {class: (p50 rel, p99 rel, max abs)}
    "bf": {"general": (4e-5, 1e-2, 4e-3), "near_parallel": (4e-5, 0.1, 2e-3), "intersecting": (2e-5, None, 2e-3)},
    "penalty": {"general": (5e-6, 5e-5, 5e-5), "near_parallel": (1e-5, 1e-4, 2e-5),
                "intersecting": (1e-5, 1e-4, 1e-5)},
    "penalty_iter": {"general": (5e-5, 1.0, 0.3), "near_parallel": (1e-4, 1.0, 0.15),
                     "intersecting": (2e-4, 1.0, 0.1)},
    "gjk": {"general": (1e-4, 2e4, 4.0), "near_parallel": (2e-4, 4e4, 4.0), "intersecting": (None, None, 4.0)},
    "hybrid": {"general": (5e-6, 5e-5, 5e-5), "near_parallel": (1e-5, 1e-4, 2e-5),
               "intersecting": (1e-5, 1e-4, 1e-5)},
}


@pytest.fixture(scope="module")
def classed_workload():
    from delta_b200.scenarios import narrowphase_pairs

    a, b, _, cls = narrowphase_pairs(1 << 17, seed=4321)
    return a, b, cls


@pytest.mark.parametrize("name", list(F32_BOUNDS))
def test_f32_methods_error_vs_f64_oracle_per_class(ctx, oracle, classed_workload, name):
    from delta_b200.scenarios import CLASS_NAMES

    a, b, cls = classed_workload
    m = METHODS[name]
    _, _, d32, _ = _run(ctx, m, a, b, precision=1)
    _, _, d64, _ = oracle.pairs(m, a, b, max_error=MAX_ERR)
    assert np.all(np.isfinite(d32))
    for c, cname in enumerate(CLASS_NAMES):
        sel = (cls == c) & np.isfinite(d64)
        err = np.abs(d32[sel] - d64[sel])
        pos = d64[sel] > 0
        rel = err[pos] / d64[sel][pos]
        p50, p99, amax = F32_BOUNDS[name][cname]
        assert err.max() <= amax, (cname, err.max())
        if p50 is not None:
            assert np.quantile(rel, 0.5) <= p50, (cname, np.quantile(rel, 0.5))
        if p99 is not None:
            assert np.quantile(rel, 0.99) <= p99, (cname, np.quantile(rel, 0.99))


def test_host_path_equals_device_path(ctx, workload):
    from delta_b200.narrowphase import pairs_host

    a, b = workload
    hp, hq, hd, hf = pairs_host(ctx, 0, a, b, max_error=MAX_ERR)
    gp, gq, gd, gf = _run(ctx, 0, a, b)
    assert np.array_equal(hp, gp) and np.array_equal(hq, gq) and np.array_equal(hd, gd)


def test_host_pipeline_many_chunks_and_pitch(ctx):
    """The host entry point streams several chunks (transfers overlapping compute); with a
    host pitch ld > n the results equal the device path and entries past n stay untouched."""
    import ctypes

    from delta_b200._lib import check, lib
    from delta_b200.narrowphase import pairs_device
    from delta_b200.scenarios import narrowphase_pairs

    n, ld = (1 << 20) + 777, (1 << 20) + 1000
    a, b, _, _ = narrowphase_pairs(n, seed=8)
    A = np.zeros((9, ld)); B = np.zeros((9, ld))
    A[:, :n] = a; B[:, :n] = b
    P = np.full((3, ld), 7.0); Q = P.copy(); D = np.full(ld, 7.0); F = np.full(ld, 9, np.uint8)
    ptr = lambda x: x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    check(lib().delta_pairs_run_host(ctx.handle, 5, 0, n, ptr(A), ptr(B), ld, 0.0, ptr(P), ptr(Q), ptr(D), ptr(F)))
    gp, gq, gd, gf = pairs_device(ctx, 5, _dev(a), _dev(b))
    ctx.synchronize()
    assert np.array_equal(P[:, :n], gp.cpu().numpy()) and np.array_equal(Q[:, :n], gq.cpu().numpy())
    assert np.array_equal(D[:n], gd.cpu().numpy()) and np.array_equal(F[:n], gf.cpu().numpy())
    assert np.all(P[:, n:] == 7.0) and np.all(D[n:] == 7.0) and np.all(F[n:] == 9)


def test_padded_leading_dimension(ctx, oracle, workload):
    """ld > n: the planes are strided; entries past n are untouched."""
    import ctypes
    import torch

    from delta_b200._lib import check, lib

    a, b = workload
    n, ld = 1000, 1536
    A = torch.zeros((9, ld), dtype=torch.float64, device="cuda")
    B = torch.zeros_like(A)
    A[:, :n] = _dev(a[:, :n]); B[:, :n] = _dev(b[:, :n])
    P = torch.full((3, ld), 7.0, dtype=torch.float64, device="cuda"); Q = P.clone()
    D = torch.full((ld,), 7.0, dtype=torch.float64, device="cuda")
    check(lib().delta_pairs_run(ctx.handle, 0, 0, n, A.data_ptr(), B.data_ptr(), ld, 0.0, P.data_ptr(),
                                Q.data_ptr(), D.data_ptr(), None))
    ctx.synchronize()
    op, oq, od, _ = oracle.pairs(0, a[:, :n], b[:, :n])
    assert np.array_equal(P[:, :n].cpu().numpy(), op) and np.array_equal(D[:n].cpu().numpy(), od)
    assert torch.all(P[:, n:] == 7.0) and torch.all(D[n:] == 7.0)


def test_empty_and_invalid_arguments(ctx):
    from delta_b200._lib import DeltaError, check, lib

    check(lib().delta_pairs_run(ctx.handle, 0, 0, 0, None, None, 0, 0.0, None, None, None, None))
    with pytest.raises(DeltaError, match="INVALID"):
        check(lib().delta_pairs_run(ctx.handle, 99, 0, 4, None, None, 4, 0.0, None, None, None, None))
    with pytest.raises(DeltaError, match="INVALID"):
        check(lib().delta_pairs_run(ctx.handle, 0, 0, 8, None, None, 4, 0.0, None, None, None, None))


def test_autotuned_launch_keeps_results(ctx, oracle, workload):
    """The autotuner picks a launch shape; results stay bit-exact with every shape."""
    from delta_b200.narrowphase import autotune, set_launch

    a, b = workload
    for m in (0, 5):
        cfg = autotune(ctx, m, _dev(a), _dev(b))
        assert cfg["threads"] in (64, 128, 256) and cfg["blocks_per_sm"] >= 0 and cfg["ms"] > 0
        gp, gq, gd, _ = _run(ctx, m, a, b)
        op, oq, od, _ = oracle.pairs(0, a, b)
        assert not (_differ(gp, op) | _differ(gq, oq) | _differ(gd[None], od[None])).any()
    # a capped grid (grid-stride loop, warps regrouped per 32 pairs) and one thread per pair
    for shape in ((64, 4), (128, 1), (128, 0)):
        set_launch(ctx, 0, 0, *shape)
        gp, gq, gd, _ = _run(ctx, 0, a, b)
        assert not (_differ(gp, op) | _differ(gq, oq) | _differ(gd[None], od[None])).any(), shape
    from delta_b200._lib import DeltaError

    with pytest.raises(DeltaError, match="INVALID"):
        set_launch(ctx, 0, 0, 256, 32)  # the FP64 bf kernel takes at most 128 threads per block
