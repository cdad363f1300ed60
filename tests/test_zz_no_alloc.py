"""The allocation-free host entry point, delta_pairs_run_host_noalloc.

Callers that cannot let the library allocate device memory (their own pool owns it,
they record work by stream capture, or they run allocation-free loops) use this entry
point; it stages through a fixed device array built into the library.  This file is
collected last so that a failure here stops a -x run only after every other test ran.
The test checks the new entry point against delta_pairs_run_host (bit for bit, the
tolerance these pair tests use) on two different inputs in a row, and that sizes above
the stated maximum are refused.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(ctx, fn, method, a, b, max_error=1e-3):
    from delta_b200._lib import check

    n = a.shape[1]
    p = np.empty((3, n)); q = np.empty((3, n)); d = np.empty(n); fl = np.empty(n, np.uint8)
    check(fn(ctx.handle, method, 0, n, a.ctypes.data, b.ctypes.data, n, max_error, p.ctypes.data, q.ctypes.data,
             d.ctypes.data, fl.ctypes.data))
    return p, q, d, fl


@pytest.mark.parametrize("method", [0, 1, 5])
def test_noalloc_matches_allocating_entry_point_twice(ctx, method):
    from delta_b200._lib import lib
    from delta_b200.scenarios import narrowphase_pairs

    L = lib()
    for seed, n in ((71, 40000), (72, 25000)):  # the second call is smaller: stale data must not leak
        a, b, _, _ = narrowphase_pairs(n, seed=seed)
        ref = _call(ctx, L.delta_pairs_run_host, method, a, b)
        new = _call(ctx, L.delta_pairs_run_host_noalloc, method, a, b)
        for x, y in zip(ref, new):
            assert np.array_equal(x, y, equal_nan=True)


def test_noalloc_rejects_sizes_above_the_maximum(ctx):
    from delta_b200._lib import DeltaError, check, lib

    n = 327680 + 1
    dummy = np.zeros(1)
    with pytest.raises(DeltaError, match="CAPACITY"):
        check(lib().delta_pairs_run_host_noalloc(ctx.handle, 0, 0, n, dummy.ctypes.data, dummy.ctypes.data, n, 0.0,
                                                 dummy.ctypes.data, dummy.ctypes.data, dummy.ctypes.data, None))
