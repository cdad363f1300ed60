"""Trains the learned warm start on the GPU and writes its checkpoint.

    python -m delta_b200.train_warmstart [--pairs-log2 26] [--epochs 20] [--batch 65536]
                                         [--lr 1e-3] [--eval-log2 24] [--out PATH]

Training pairs are the narrowphase microbenchmark's distribution (scenarios.narrowphase_pairs),
labelled by the FP64 bfSolver kernel; the network is trained with the library's own
forward, backward and Adam kernels.  The evaluation set is a fresh draw: it reports the
loss, the reference penalty iteration's mean iteration count from the prediction versus
from 0.33, and the learned solver's certified fraction with and without the network.
The checkpoint is an .npz (FP32 parameters in the library's flat layout) with a .json
summary beside it.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

DEFAULT_OUT = Path(__file__).resolve().parent / "weights" / "warmstart_mlp.npz"
CHUNK_LOG2 = 22


def _pairs(n, seed):
    from .scenarios import narrowphase_pairs_chunked

    return narrowphase_pairs_chunked(n, seed=seed)[:2]


def build_training_set(ctx, n, seed):
    """(X, T, valid) on the device for n fresh pairs, generated and labelled in chunks."""
    import torch

    from .learned import labelled

    chunk = min(n, 1 << CHUNK_LOG2)
    X = torch.empty((n, 32), dtype=torch.bfloat16, device="cuda")
    T = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    V = torch.empty(n, dtype=torch.uint8, device="cuda")
    for k, s in enumerate(range(0, n, chunk)):
        a, b = _pairs(min(chunk, n - s), seed + 104729 * k)
        x, t, v = labelled(ctx, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
        X[s:s + x.shape[0]] = x
        T[s:s + x.shape[0]] = t
        V[s:s + x.shape[0]] = v
    return X, T, V


def evaluate(ctx, model, n, seed):
    import torch

    from ._lib import check, lib
    from .learned import labelled, learned_pairs

    a_np, b_np = _pairs(n, seed)
    a, b = torch.from_numpy(a_np).cuda(), torch.from_numpy(b_np).cuda()
    X, T, V = labelled(ctx, a, b)
    out = {"pairs": n}
    # loss over the evaluation set, in batches
    tot, nv = 0.0, 0
    for s in range(0, n, 1 << 20):
        Y = model.forward(X[s:s + (1 << 20)])
        v = V[s:s + (1 << 20)].bool()
        tot += float(((Y - T[s:s + (1 << 20)]) ** 2).sum(1)[v].sum().item())
        nv += int(v.sum().item())
    out["loss"] = tot / max(nv, 1)
    x0 = model.predict(a, b)
    for name, start in (("network", x0), ("plain", None)):
        p = torch.empty((3, n), dtype=torch.float64, device="cuda")
        q, d = torch.empty_like(p), torch.empty(n, dtype=torch.float64, device="cuda")
        it = torch.empty(n, dtype=torch.uint8, device="cuda")
        check(lib().delta_penalty_warm(ctx.handle, n, a.data_ptr(), b.data_ptr(), n,
                                       None if start is None else start.data_ptr(), 1e-6, p.data_ptr(), q.data_ptr(),
                                       d.data_ptr(), it.data_ptr()))
        out[f"penalty_mean_iterations_{name}"] = float(it.float().mean().item())
    for sweeps in (0, 1, 2, 4):
        for name, m in (("network", model), ("plain", None)):
            nf = learned_pairs(ctx, m, a, b, sweeps=sweeps, count_fallback=True)[4]
            out[f"certified_fraction_{name}_sweeps{sweeps}"] = 1.0 - nf / n
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs-log2", type=int, default=26)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval-log2", type=int, default=24)
    ap.add_argument("--seed", type=int, default=20260)
    ap.add_argument("--out", default=str(DEFAULT_OUT))
    args = ap.parse_args(argv)

    import torch

    from .learned import WarmStartMLP, train
    from .narrowphase import Context

    ctx = Context(0)
    t0 = time.perf_counter()
    X, T, V = build_training_set(ctx, 1 << args.pairs_log2, args.seed)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    model = WarmStartMLP(ctx, seed=args.seed)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    losses = train(model, X, T, V, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=args.seed,
                   log=lambda m: print(m, flush=True))
    e.record()
    torch.cuda.synchronize()
    train_s = s.elapsed_time(e) / 1e3
    samples = args.epochs * (X.shape[0] // args.batch) * args.batch
    del X, T, V
    ev = evaluate(ctx, model, 1 << args.eval_log2, args.seed + 1)
    out = Path(args.out)
    out.parent.mkdir(parents=True, exist_ok=True)
    np.savez(out, params=model.params.cpu().numpy())
    summary = {
        "architecture": "18 (padded to 32) -> 128 -> 128 -> 128 -> 4, GELU (tanh form), BF16 weights and activations, "
                        "FP32 accumulation; Adam on FP32 master weights",
        "training_pairs": 1 << args.pairs_log2, "epochs": args.epochs, "batch": args.batch, "lr": args.lr,
        "seed": args.seed, "epoch_loss": losses, "train_seconds": train_s,
        "train_samples_per_second": samples / train_s, "data_seconds": t_data,
        "evaluation": ev,
        "device": torch.cuda.get_device_name(0),
        "gemm_engine": getattr(ctx, "mlp_engine", "tcgen05"),
    }
    out.with_suffix(".json").write_text(json.dumps(summary, indent=1) + "\n")
    print(json.dumps(summary, indent=1))
    ctx.close()


if __name__ == "__main__":
    main()
