"""CPU restatement of the learned warm start's arithmetic (test infrastructure, not the
product).  Only tests/ import this module.

The network has no counterpart in the reference; its inputs and targets do: the targets
are barycentric weights of bfSolver's closest points (bf.cpp:217-1178) in the
parametrisation penaltySolver uses (P = A0 + x0 (A1-A0) + x1 (A2-A0), penalty.cpp:353-356
start x = 0.33).  This module restates, in numpy:

* ``canon``: the canonical features and targets, operation for operation as the CUDA
  path computes them (each FP64 operation rounded once, then FP32, then BF16), so the
  features agree bit for bit;
* ``forward`` / ``backward``: the MLP and the gradient of its MSE loss, accumulating in
  FP64.  With ``rounded=True`` the BF16 roundings the CUDA path applies (weights,
  activations, output and hidden gradients) are mirrored, so the remaining difference is
  FP32 versus FP64 accumulation; with ``rounded=False`` it is plain FP64 calculus, for
  finite-difference checks;
* ``adam``: one bias-corrected Adam step (Kingma & Ba 2015).
"""
from __future__ import annotations

import numpy as np

IN, HIDDEN, OUT, FEATURES = 32, 128, 4, 18
LAYERS = ((IN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, OUT))


def layout() -> dict:
    """Offsets of W1, b1, ..., W4, b4 in the flat parameter array, and its padded length."""
    off, o = {}, 0
    for l, (fi, fo) in enumerate(LAYERS, start=1):
        off[f"W{l}"] = o
        o += fo * fi
        off[f"b{l}"] = o
        o += fo
    off["total"] = (o + 7) // 8 * 8
    return off


def unpack(flat: np.ndarray) -> dict:
    L = layout()
    out = {}
    for l, (fi, fo) in enumerate(LAYERS, start=1):
        out[f"W{l}"] = flat[L[f"W{l}"]:L[f"W{l}"] + fo * fi].reshape(fo, fi)
        out[f"b{l}"] = flat[L[f"b{l}"]:L[f"b{l}"] + fo]
    return out


def pack(d: dict) -> np.ndarray:
    L = layout()
    flat = np.zeros(L["total"], np.float64)
    for l in range(1, 5):
        flat[L[f"W{l}"]:L[f"W{l}"] + d[f"W{l}"].size] = d[f"W{l}"].ravel()
        flat[L[f"b{l}"]:L[f"b{l}"] + d[f"b{l}"].size] = d[f"b{l}"]
    return flat


def bf16(x) -> np.ndarray:
    """Round to BF16 (nearest, ties to even) through FP32; returns float64 values."""
    u = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _dot3(a, b):
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]


def _cross(u, v):
    return np.stack([u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]])


def canon(a: np.ndarray, b: np.ndarray, p: np.ndarray | None = None, q: np.ndarray | None = None):
    """Features (n, 32) as BF16 values, targets (n, 4) FP32 or None, valid (n,) bool.

    a, b: pair-list planes (9, n) float64; p, q: closest points (3, n)."""
    A = [a[3 * v:3 * v + 3] for v in range(3)]
    B = [b[3 * v:3 * v + 3] for v in range(3)]
    n = a.shape[1]
    with np.errstate(divide="ignore", invalid="ignore"):
        c = ((A[0] + A[1]) + A[2]) / 3.0
        E0, E1, E2, E3 = A[1] - A[0], A[2] - A[0], A[2] - A[1], A[0] - A[2]
        nr = _cross(E0, E1)
        l0, l1, l2 = np.sqrt(_dot3(E0, E0)), np.sqrt(_dot3(E2, E2)), np.sqrt(_dot3(E3, E3))
        ln = np.sqrt(_dot3(nr, nr))
        emax = l0.copy()
        emax = np.where(l1 > emax, l1, emax)
        emax = np.where(l2 > emax, l2, emax)
        ok = (l0 > 0) & (ln > 0)
        e1 = np.where(ok, E0 / l0, 0.0)
        e3 = np.where(ok, nr / ln, 0.0)
        e2 = _cross(e3, e1)
        s = np.where(ok, 1.0 / emax, 0.0)
        f = np.zeros((n, IN), np.float64)
        for v, X in enumerate(A + B):
            d = X - c
            for k, e in enumerate((e1, e2, e3)):
                f[:, 3 * v + k] = bf16((s * _dot3(d, e)).astype(np.float32))
        T = None
        if p is not None:
            T = np.zeros((n, OUT), np.float32)
            x = []
            for Tri, src in ((A, p), (B, q)):
                U, V, W = Tri[1] - Tri[0], Tri[2] - Tri[0], src - Tri[0]
                uu, uv, vv, wu, wv = _dot3(U, U), _dot3(U, V), _dot3(V, V), _dot3(W, U), _dot3(W, V)
                det = uu * vv - uv * uv
                ok = ok & (det > (1e-12 * uu) * vv)
                x += [(wu * vv - wv * uv) / det, (wv * uu - wu * uv) / det]
            for k in range(4):
                T[:, k] = np.where(ok, x[k], 0.0).astype(np.float32)
    return f, T, ok


_K = np.sqrt(2.0 / np.pi)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(_K * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    th = np.tanh(_K * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * _K * (1.0 + 3 * 0.044715 * x * x)


def forward(X: np.ndarray, params: dict, rounded: bool = True) -> dict:
    """X (M, 32); params from unpack().  Returns the cache (Z1..Z3, H0..H3, Y)."""
    r = bf16 if rounded else (lambda v: np.asarray(v, np.float64))
    cache = {"H0": np.asarray(X, np.float64)}
    h = cache["H0"]
    for l in range(1, 5):
        W = r(params[f"W{l}"])
        z = h @ W.T + np.asarray(params[f"b{l}"], np.float64)
        if l < 4:
            if rounded:
                z = z.astype(np.float32).astype(np.float64)
            cache[f"Z{l}"] = z
            h = r(gelu(z))
            cache[f"H{l}"] = h
        else:
            cache["Y"] = z
    return cache


def backward(cache: dict, params: dict, T: np.ndarray, valid: np.ndarray, rounded: bool = True):
    """Loss and gradients (dict like params) of mean over valid rows of sum (Y - T)^2."""
    r = bf16 if rounded else (lambda v: np.asarray(v, np.float64))
    n = max(int(valid.sum()), 1)
    diff = np.where(valid[:, None], cache["Y"] - T, 0.0)
    loss = float((diff ** 2).sum() / n)
    d = r(2.0 * diff / n)
    g = {}
    for l in range(4, 0, -1):
        g[f"W{l}"] = d.T @ cache[f"H{l - 1}"]
        g[f"b{l}"] = d.sum(0)
        if l == 1:
            break
        dh = d @ r(params[f"W{l}"])
        d = r(dh * gelu_grad(cache[f"Z{l - 1}"]))
    return loss, g


def adam(w, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step on float64 copies; returns (w, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return w, m, v
