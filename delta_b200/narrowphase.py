"""Pair-list narrowphase: closest points of independent triangle pairs.

Mirrors the reference's per-pair solvers (delta/contact/detection):
``bfSolver`` (bf.cpp:217), ``penaltySolver`` with a failure flag (penalty.cpp:278) or an
iteration count (penalty.cpp:434), ``gjk(a,3,b,3,p,q)`` (gjk.cpp:418), applied to a
structure-of-arrays pair list in the shape of ``ispc_bf``/``ispc_pen`` (bf.ispc:3,
penalty.ispc:154).  All work runs in libdelta_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib

BF, PENALTY, PENALTY_ITER, GJK, HYBRID_PAIR, BF_CERT = range(6)
F64, F32 = 0, 1
METHODS = {"bf": BF, "penalty": PENALTY, "penalty_iter": PENALTY_ITER, "gjk": GJK, "hybrid": HYBRID_PAIR,
           "bf_cert": BF_CERT}


class Context:
    """A delta_ctx on one device, bound to a CUDA stream (default: torch's current)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._h = C.c_void_p()
        if stream is None:
            try:
                import torch

                if torch.cuda.is_available():
                    stream = torch.cuda.current_stream(device).cuda_stream
            except ImportError:
                stream = None
        check(lib().delta_create(C.byref(self._h), device, C.c_void_p(stream or 0)))
        self.device = device

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream: int):
        check(lib().delta_set_stream(self._h, C.c_void_p(stream)))

    def synchronize(self):
        check(lib().delta_synchronize(self._h))

    def set_cull_launch(self, cull_blocks_per_sm: int, survivor_blocks_per_sm: int):
        """Blocks per SM of the culled drivers' culling and survivor kernels (0 = all that fit)."""
        check(lib().delta_set_cull_launch(self._h, int(cull_blocks_per_sm), int(survivor_blocks_per_sm)))

    @property
    def launches(self) -> int:
        return int(lib().delta_launch_count(self._h))

    def close(self):
        if self._h:
            lib().delta_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _method(m) -> int:
    return METHODS[m] if isinstance(m, str) else int(m)


def pairs_device(ctx: Context, method, a, b, out=None, precision=F64, max_error=0.0, with_flags=True):
    """Runs on CUDA tensors a, b of shape (9, n) float64 (plane 3*vertex+coord).

    Returns (p, q, dist, flags) as CUDA tensors; asynchronous on the context's stream.
    """
    import torch

    if a.dtype != torch.float64 or b.dtype != torch.float64 or not a.is_cuda or not b.is_cuda:
        raise TypeError("a, b must be float64 CUDA tensors")
    if a.shape != b.shape or a.shape[0] != 9:
        raise ValueError("a, b must have shape (9, n)")
    a = a.contiguous(); b = b.contiguous()
    n = a.shape[1]
    if out is None:
        p = torch.empty((3, n), dtype=torch.float64, device=a.device)
        q = torch.empty_like(p)
        d = torch.empty(n, dtype=torch.float64, device=a.device)
        fl = torch.empty(n, dtype=torch.uint8, device=a.device) if with_flags else None
    else:
        p, q, d, fl = out
    check(lib().delta_pairs_run(ctx.handle, _method(method), int(precision), n, a.data_ptr(), b.data_ptr(), n,
                                float(max_error), p.data_ptr(), q.data_ptr(), d.data_ptr(),
                                fl.data_ptr() if fl is not None else None))
    return p, q, d, fl


def pairs_host(ctx: Context, method, a: np.ndarray, b: np.ndarray, out=None, precision=F64, max_error=0.0,
               with_flags=True):
    """Host arrays in, host arrays out (copies to and from the device inside; synchronous)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    if a.shape != b.shape or a.shape[0] != 9:
        raise ValueError("a, b must have shape (9, n)")
    n = a.shape[1]
    if out is None:
        p = np.empty((3, n)); q = np.empty((3, n)); d = np.empty(n)
        fl = np.empty(n, np.uint8) if with_flags else None
    else:
        p, q, d, fl = out
    ptr = lambda x: None if x is None else x.ctypes.data  # noqa: E731
    check(lib().delta_pairs_run_host(ctx.handle, _method(method), int(precision), n, ptr(a), ptr(b), n,
                                     float(max_error), ptr(p), ptr(q), ptr(d), ptr(fl)))
    return p, q, d, fl


def autotune(ctx: Context, method, a, b, precision=F64, max_error=0.0, out=None):
    """Times the candidate launch shapes of `method` on CUDA tensors a, b (9, n) and keeps
    the fastest on `ctx`.  Returns {"threads", "blocks_per_sm", "ms"}."""
    import torch

    n = a.shape[1]
    if out is None:
        out = (torch.empty((3, n), dtype=torch.float64, device=a.device),
               torch.empty((3, n), dtype=torch.float64, device=a.device),
               torch.empty(n, dtype=torch.float64, device=a.device), torch.empty(n, dtype=torch.uint8, device=a.device))
    p, q, d, fl = out
    t = C.c_int32(0); bps = C.c_int32(0); ms = C.c_float(0)
    check(lib().delta_autotune_pairs(ctx.handle, _method(method), int(precision), n, a.data_ptr(), b.data_ptr(), n,
                                     float(max_error), p.data_ptr(), q.data_ptr(), d.data_ptr(), fl.data_ptr(),
                                     C.byref(t), C.byref(bps), C.byref(ms)))
    return {"threads": t.value, "blocks_per_sm": bps.value, "ms": ms.value}


def set_launch(ctx: Context, method, precision, threads: int, blocks_per_sm: int):
    check(lib().delta_set_pair_launch(ctx.handle, _method(method), int(precision), int(threads), int(blocks_per_sm)))
