"""Learned warm start for the triangle-pair narrowphase.

A small MLP maps a canonicalised triangle pair (triangle A's frame, unit = its longest
edge: 18 coordinates) to the barycentric weights of the closest points, the four
parameters penaltySolver iterates on and starts at 0.33 (penalty.cpp:353-356).  It is
trained on the GPU with the library's own kernels (BF16 tensor-core GEMMs, GELU,
MSE, Adam in libdelta_b200.so); torch only holds the device memory.  Labels are the
FP64 bfSolver closest points (bf.cpp:217-1178) of the same pairs.

The learned solver (`learned_pairs`) starts from the prediction, identifies the
closest features, evaluates them in FP64 with the reference arithmetic, certifies the
distance with a separating plane, and sends every uncertified pair to DELTA_BF_CERT,
which is exact; the brute force is both the fallback and the reference for the error.  There is no
counterpart of this module in the reference.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import check, lib
from .narrowphase import BF, F64, Context, pairs_device

IN, HIDDEN, OUT, FEATURES = 32, 128, 4, 18
LAYERS = ((IN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, OUT))  # (fan_in, fan_out)


def default_weights():
    """Path of the checkpoint shipped with the package (trained by train_warmstart)."""
    from pathlib import Path

    return Path(__file__).resolve().parent / "weights" / "warmstart_mlp.npz"


def layout() -> dict:
    """Flat parameter layout from the library: offsets of W1, b1, ..., W4, b4 and the total."""
    off = (C.c_int64 * 9)()
    check(lib().delta_mlp_layout(off))
    names = ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4", "total")
    return dict(zip(names, [int(x) for x in off]))


def init_params(seed: int = 0) -> np.ndarray:
    """FP32 initial parameters in the flat layout: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for
    weights and biases (fan_in of layer 1 = the 18 used features; its padding columns 0)."""
    L = layout()
    rng = np.random.default_rng(seed)
    w = np.zeros(L["total"], np.float32)
    for l, (fi, fo) in enumerate(LAYERS, start=1):
        used = FEATURES if l == 1 else fi
        bound = 1.0 / math.sqrt(used)
        W = np.zeros((fo, fi), np.float32)
        W[:, :used] = rng.uniform(-bound, bound, (fo, used))
        w[L[f"W{l}"]:L[f"W{l}"] + fo * fi] = W.ravel()
        w[L[f"b{l}"]:L[f"b{l}"] + fo] = rng.uniform(-bound, bound, fo)
    return w


class WarmStartMLP:
    """18 -> 128 -> 128 -> 128 -> 4 with GELU, BF16 weights/activations, FP32 master
    weights and Adam moments, on one context's device."""

    def __init__(self, ctx: Context, seed: int = 0, params: np.ndarray | None = None):
        import torch

        self.ctx = ctx
        self.L = layout()
        self.dev = torch.device("cuda", ctx.device)
        host = init_params(seed) if params is None else np.asarray(params, np.float32)
        if host.shape != (self.L["total"],):
            raise ValueError(f"params must have {self.L['total']} entries")
        self.params = torch.from_numpy(host.copy()).to(self.dev)
        self.params_bf16 = torch.empty(self.L["total"], dtype=torch.bfloat16, device=self.dev)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.steps = 0
        self._ws_rows = 0
        self._refresh_bf16()

    # -- parameter views ---------------------------------------------------------------
    def _view(self, t, name, shape):
        o = self.L[name]
        return t[o:o + int(np.prod(shape))].view(*shape)

    def weight(self, l, bf16=True):
        fi, fo = LAYERS[l - 1]
        return self._view(self.params_bf16 if bf16 else self.params, f"W{l}", (fo, fi))

    def bias(self, l):
        return self._view(self.params, f"b{l}", (LAYERS[l - 1][1],))

    def grad(self, name):
        l = int(name[1])
        fi, fo = LAYERS[l - 1]
        return self._view(self.grads, name, (fo, fi) if name[0] == "W" else (fo,))

    def _refresh_bf16(self):
        check(lib().delta_to_bf16(self.ctx.handle, self.L["total"], self.params.data_ptr(),
                                  self.params_bf16.data_ptr()))

    def state_dict(self) -> dict:
        return {"params": self.params.cpu().numpy(), "steps": self.steps}

    @classmethod
    def load(cls, ctx: Context, path=None) -> "WarmStartMLP":
        """A network from a checkpoint written by train_warmstart (default: the bundled one)."""
        from pathlib import Path

        p = Path(path) if path is not None else default_weights()
        with np.load(p) as z:
            return cls(ctx, params=z["params"])

    # -- workspace ---------------------------------------------------------------------
    def _workspace(self, M):
        import torch

        if self._ws_rows >= M:
            return
        f32 = dict(dtype=torch.float32, device=self.dev)
        b16 = dict(dtype=torch.bfloat16, device=self.dev)
        self.Z = [torch.empty((M, HIDDEN), **f32) for _ in range(3)]
        self.H = [torch.empty((M, HIDDEN), **b16) for _ in range(3)]
        self.Y = torch.empty((M, OUT), **f32)
        self.dY = torch.empty((M, OUT), **b16)
        self.dH = torch.empty((M, HIDDEN), **f32)
        self.dZ = torch.empty((M, HIDDEN), **b16)
        self.loss = torch.zeros(1, **f32)
        self._ws_rows = M

    # -- kernels -----------------------------------------------------------------------
    def _gemm(self, M, N, K, A, lda, ta, B, ldb, tb, Cm, ldc, acc=0, split=1):
        check(lib().delta_gemm_bf16(self.ctx.handle, M, N, K, A.data_ptr(), lda, ta, B.data_ptr(), ldb, tb,
                                    Cm.data_ptr(), ldc, acc, split))

    def forward(self, X):
        """Layer by layer on X (M, 32) BF16; returns Y (M, 4) FP32 (a workspace view)."""
        M = X.shape[0]
        self._workspace(M)
        h = X
        for l in range(1, 4):
            fi = LAYERS[l - 1][0]
            Z, H = self.Z[l - 1][:M], self.H[l - 1][:M]
            self._gemm(M, HIDDEN, fi, h, fi, 0, self.weight(l), fi, 1, Z, HIDDEN)
            check(lib().delta_mlp_bias_act(self.ctx.handle, M, HIDDEN, Z.data_ptr(), self.bias(l).data_ptr(),
                                           H.data_ptr(), 1))
            h = H
        Y = self.Y[:M]
        self._gemm(M, OUT, HIDDEN, h, HIDDEN, 0, self.weight(4), HIDDEN, 1, Y, OUT)
        check(lib().delta_mlp_bias_act(self.ctx.handle, M, OUT, Y.data_ptr(), self.bias(4).data_ptr(), None, 0))
        return Y

    def backward(self, X, T, valid, n_valid: int):
        """Gradients of the MSE over valid rows into self.grads (after forward(X))."""
        M = X.shape[0]
        # split-K of the weight gradients (K = the batch): the tcgen05 GEMM adds the partial
        # tiles in a second kernel; about two CTAs per SM (one left the SM's loads
        # latency-bound), each with K/split >= 256 rows so that its two-buffer pipeline
        # runs several chunks
        if getattr(self.ctx, "mlp_engine", "tcgen05") == "tcgen05":
            split = max(1, min(296, M // 256))
        else:
            split = max(1, min(128, M // 1024))
        self.grads.zero_()
        self.loss.zero_()
        h = lib()
        dY = self.dY[:M]
        check(h.delta_mlp_mse(self.ctx.handle, M, self.Y[:M].data_ptr(), T.data_ptr(), valid.data_ptr(),
                              1.0 / max(n_valid, 1), dY.data_ptr(), self.loss.data_ptr()))
        d, width = dY, OUT
        for l in range(4, 0, -1):
            fi, fo = LAYERS[l - 1]
            prev = X if l == 1 else self.H[l - 2][:M]
            # dW[fo, fi] = d^T prev ; db = column sums of d
            self._gemm(fo, fi, M, d, width, 1, prev, fi, 0, self.grad(f"W{l}"), fi, 1, split)
            check(h.delta_mlp_colsum(self.ctx.handle, M, fo, d.data_ptr(), self.grad(f"b{l}").data_ptr()))
            if l == 1:
                break
            dH = self.dH[:M]
            self._gemm(M, fi, fo, d, width, 0, self.weight(l), fi, 0, dH, fi)
            dZ = self.dZ[:M]
            check(h.delta_mlp_act_grad(self.ctx.handle, M, fi, dH.data_ptr(), self.Z[l - 2][:M].data_ptr(),
                                       dZ.data_ptr()))
            d, width = dZ, fi

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.steps += 1
        check(lib().delta_adam(self.ctx.handle, self.L["total"], self.params.data_ptr(), self.grads.data_ptr(),
                               self.m.data_ptr(), self.v.data_ptr(), lr, b1, b2, eps, self.steps,
                               self.params_bf16.data_ptr()))

    def train_step(self, X, T, valid, n_valid: int, lr=1e-3):
        self.forward(X)
        self.backward(X, T, valid, n_valid)
        self.adam(lr)

    # -- inference ---------------------------------------------------------------------
    def predict(self, a, b, out=None, engine: str = "mma"):
        """x0 (n, 4) FP32 for pair-list tensors a, b (9, n) on the device: the features
        kernel and one fused network kernel, on the mma.sync tensor-core path ("mma") or
        the tcgen05/TMEM path ("tcgen05", synchronous)."""
        import torch

        n = a.shape[1]
        x0 = out if out is not None else torch.empty((n, OUT), dtype=torch.float32, device=a.device)
        fn = lib().delta_mlp_infer_tcgen05 if engine == "tcgen05" else lib().delta_mlp_infer
        check(fn(self.ctx.handle, n, a.data_ptr(), b.data_ptr(), a.stride(0), self.params.data_ptr(),
                 self.params_bf16.data_ptr(), x0.data_ptr()))
        return x0


ENGINES = {"tcgen05": 0, "mma": 1}


def set_engine(ctx: Context, engine: str):
    """Network engine of the learned hybrid on this context: "tcgen05" (default) or "mma"."""
    check(lib().delta_mlp_set_engine(ctx.handle, ENGINES[engine]))
    ctx.mlp_engine = engine


def features(ctx: Context, a, b, p=None, q=None):
    """(X (n, 32) BF16, T (n, 4) FP32 or None, valid (n,) uint8) for pair-list tensors."""
    import torch

    n = a.shape[1]
    X = torch.empty((n, IN), dtype=torch.bfloat16, device=a.device)
    T = torch.empty((n, OUT), dtype=torch.float32, device=a.device) if p is not None else None
    valid = torch.empty(n, dtype=torch.uint8, device=a.device)
    check(lib().delta_mlp_features(ctx.handle, n, a.data_ptr(), b.data_ptr(), a.stride(0),
                                   None if p is None else p.data_ptr(), None if q is None else q.data_ptr(),
                                   X.data_ptr(), None if T is None else T.data_ptr(), valid.data_ptr()))
    return X, T, valid


def labelled(ctx: Context, a, b):
    """Training rows for pair-list tensors a, b: features, bfSolver targets, valid flags."""
    p, q, _, _ = pairs_device(ctx, BF, a, b, precision=F64, with_flags=False)
    return features(ctx, a, b, p, q)


def train(model: WarmStartMLP, X, T, valid, epochs: int = 1, batch: int = 65536, lr: float = 1e-3,
          seed: int = 0, log=None) -> list[float]:
    """Adam over shuffled mini-batches; returns the mean loss of each epoch."""
    import torch

    n = X.shape[0]
    gen = torch.Generator(device=X.device)
    gen.manual_seed(seed)
    losses = []
    nb = n // batch
    if nb == 0:
        raise ValueError("fewer rows than one batch")
    for ep in range(epochs):
        # one gather per epoch into shuffled copies; the mini-batches are contiguous slices
        perm = torch.randperm(n, device=X.device, generator=gen)[: nb * batch]
        Xs, Ts, vb = X[perm], T[perm], valid[perm].view(nb, batch)
        del perm
        counts = vb.sum(1, dtype=torch.int64).cpu().tolist()
        total = torch.zeros(1, dtype=torch.float32, device=X.device)
        for k in range(nb):
            rows = slice(k * batch, (k + 1) * batch)
            model.train_step(Xs[rows], Ts[rows], vb[k], counts[k], lr)
            total += model.loss
        del Xs, Ts
        losses.append(float(total.item()) / nb)
        if log:
            log(f"epoch {ep}: loss {losses[-1]:.6g}")
    return losses


def refine(ctx: Context, a, b, x0=None, sweeps: int = 2, rel_tol: float = 1e-6, out=None, features: int = 3):
    """delta_learned_refine: (p, q, dist, certified) for pair-list tensors a, b."""
    import torch

    n = a.shape[1]
    if out is None:
        p = torch.empty((3, n), dtype=torch.float64, device=a.device)
        q = torch.empty_like(p)
        d = torch.empty(n, dtype=torch.float64, device=a.device)
        cert = torch.empty(n, dtype=torch.uint8, device=a.device)
    else:
        p, q, d, cert = out
    check(lib().delta_learned_refine(ctx.handle, n, a.data_ptr(), b.data_ptr(), a.stride(0),
                                     None if x0 is None else x0.data_ptr(), int(sweeps), int(features), float(rel_tol),
                                     p.data_ptr(), q.data_ptr(), d.data_ptr(), cert.data_ptr()))
    return p, q, d, cert


def learned_pairs(ctx: Context, model: WarmStartMLP | None, a, b, sweeps: int = 2, rel_tol: float = 1e-6,
                  out=None, count_fallback: bool = False, features: int = 3):
    """The learned hybrid (delta_pairs_run_learned) over pair-list tensors a, b (9, n)
    float64 on the device.

    model None runs the same solver from the centroids (the method without the network).
    Returns (p, q, dist, flags[, n_fallback]): flags 1 = certified, the distance within
    rel_tol of the exact one; 2 = solved by DELTA_BF_CERT, equal to bfSolver bit for bit.
    """
    import torch

    n = a.shape[1]
    if out is None:
        p = torch.empty((3, n), dtype=torch.float64, device=a.device)
        q = torch.empty_like(p)
        d = torch.empty(n, dtype=torch.float64, device=a.device)
        fl = torch.empty(n, dtype=torch.uint8, device=a.device)
    else:
        p, q, d, fl = out
    nf = C.c_int64(0)
    check(lib().delta_pairs_run_learned(
        ctx.handle, n, a.data_ptr(), b.data_ptr(), a.stride(0),
        None if model is None else model.params.data_ptr(), None if model is None else model.params_bf16.data_ptr(),
        int(sweeps), int(features), float(rel_tol), p.data_ptr(), q.data_ptr(), d.data_ptr(),
        None if fl is None else fl.data_ptr(), C.byref(nf) if count_fallback else None))
    if count_fallback:
        return p, q, d, fl, int(nf.value)
    return p, q, d, fl


def learned_pairs_host(ctx: Context, model: WarmStartMLP | None, a: np.ndarray, b: np.ndarray, sweeps: int = 1,
                       rel_tol: float = 1e-6, out=None, features: int = 3):
    """learned_pairs with host arrays (9, n) in and (p, q, dist, flags, n_fallback) out
    (delta_pairs_run_learned_host: copies to and from the device inside; synchronous)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    if a.shape != b.shape or a.shape[0] != 9:
        raise ValueError("a, b must have shape (9, n)")
    n = a.shape[1]
    if out is None:
        p, q, d, fl = np.empty((3, n)), np.empty((3, n)), np.empty(n), np.empty(n, np.uint8)
    else:
        p, q, d, fl = out
    nf = C.c_int64(0)
    check(lib().delta_pairs_run_learned_host(
        ctx.handle, n, a.ctypes.data, b.ctypes.data, n, None if model is None else model.params.data_ptr(),
        None if model is None else model.params_bf16.data_ptr(), int(sweeps), int(features), float(rel_tol),
        p.ctypes.data,
        q.ctypes.data, d.ctypes.data, None if fl is None else fl.ctypes.data, C.byref(nf)))
    return p, q, d, fl, int(nf.value)


def tune(ctx: Context, model: WarmStartMLP | None, a, b, sweeps=(0, 1, 2), features=(3, 7, 11, 15), reps: int = 3):
    """The learned solver's autotuner: times delta_pairs_run_learned on device pairs a, b
    for each (network on/off, sweeps, candidate features) with CUDA events and returns the
    configurations sorted fastest first ({"network", "sweeps", "features", "ms",
    "certified_fraction"})."""
    import torch

    n = a.shape[1]
    out = (torch.empty((3, n), dtype=torch.float64, device=a.device), torch.empty((3, n), dtype=torch.float64,
                                                                                  device=a.device),
           torch.empty(n, dtype=torch.float64, device=a.device), torch.empty(n, dtype=torch.uint8, device=a.device))
    stream = torch.cuda.current_stream(a.device)
    res = []
    for net in ((True, False) if model is not None else (False,)):
        for s in sweeps:
            for f in features:
                m = model if net else None
                nf = learned_pairs(ctx, m, a, b, s, out=out, count_fallback=True, features=f)[4]
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(reps):
                    learned_pairs(ctx, m, a, b, s, out=out, features=f)
                e1.record(stream)
                e1.synchronize()
                res.append({"network": net, "sweeps": s, "features": f, "ms": e0.elapsed_time(e1) / reps,
                            "certified_fraction": 1.0 - nf / n})
    return sorted(res, key=lambda r: r["ms"])
