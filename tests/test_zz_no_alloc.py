"""The allocation-free host entry point, delta_pairs_run_host_noalloc.

Some callers cannot let this library allocate device memory: a host whose own pooling
allocator owns the GPU's memory (a raw cudaMalloc there fails or fragments its pool), or
a loop that must not pay for an allocation.  They use this entry point, which stages
inputs and outputs in a fixed device array built into the library.

This file is collected last, so that a failure here stops a -x run only after every
other test ran.  It checks, through the C ABI:
- the results equal delta_pairs_run_host's bit for bit (the tolerance of these pair
  tests), for FP64 and FP32 and four methods, on two different inputs in a row (the
  second one smaller, so stale entries of the shared array would show);
- the calls allocate no device memory (free device memory is unchanged across them);
- n equal to DELTA_NOALLOC_MAX_PAIRS runs and n one above it is refused.
It passes alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(m, prec) for m in (0, 1, 3, 5) for prec in (0, 1) if not (m == 5 and prec == 1)]


def _call(ctx, fn, method, precision, a, b, max_error=1e-3):
    from delta_b200._lib import check

    n = a.shape[1]
    p = np.empty((3, n)); q = np.empty((3, n)); d = np.empty(n); fl = np.empty(n, np.uint8)
    check(fn(ctx.handle, method, precision, n, a.ctypes.data, b.ctypes.data, n, max_error, p.ctypes.data,
             q.ctypes.data, d.ctypes.data, fl.ctypes.data))
    return p, q, d, fl


def _free_bytes():
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


def test_noalloc_matches_allocating_entry_point_twice_without_allocating(ctx):
    from delta_b200._lib import lib
    from delta_b200.scenarios import narrowphase_pairs

    L = lib()
    inputs = [narrowphase_pairs(n, seed=seed)[:2] for seed, n in ((71, 40000), (72, 25000))]
    refs = {(c, k): _call(ctx, L.delta_pairs_run_host, *c, a, b) for c in CASES for k, (a, b) in enumerate(inputs)}
    for c in CASES:  # first calls: the array's address lookup and the module/kernel loads
        _call(ctx, L.delta_pairs_run_host_noalloc, *c, *inputs[1])
    free0 = _free_bytes()
    for c in CASES:
        for k, (a, b) in enumerate(inputs):  # two calls in a row, the second smaller
            new = _call(ctx, L.delta_pairs_run_host_noalloc, *c, a, b)
            for x, y in zip(refs[(c, k)], new):
                assert np.array_equal(x, y, equal_nan=True), (c, k)
    assert _free_bytes() == free0, "a no-alloc call changed the free device memory"


def test_noalloc_maximum_size_runs_and_one_more_is_refused(ctx):
    from delta_b200._lib import DeltaError, check, header_define, lib
    from delta_b200.scenarios import narrowphase_pairs

    nmax = header_define("DELTA_NOALLOC_MAX_PAIRS")
    a, b = narrowphase_pairs(nmax, seed=73)[:2]
    ref = _call(ctx, lib().delta_pairs_run_host, 5, 0, a, b)
    new = _call(ctx, lib().delta_pairs_run_host_noalloc, 5, 0, a, b)
    for x, y in zip(ref, new):
        assert np.array_equal(x, y, equal_nan=True)
    n = nmax + 1
    dummy = np.zeros(1)
    with pytest.raises(DeltaError, match="CAPACITY"):
        check(lib().delta_pairs_run_host_noalloc(ctx.handle, 0, 0, n, dummy.ctypes.data, dummy.ctypes.data, n, 0.0,
                                                 dummy.ctypes.data, dummy.ctypes.data, dummy.ctypes.data, None))
