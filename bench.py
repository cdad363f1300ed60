#!/usr/bin/env python
"""Benchmark of the B200 contact narrowphase (one JSON line on rank 0).

Workload: the narrowphase microbenchmark, 2^24 independent triangle pairs (triangle A
~ U[0,1]^3, B a rotated triangle with edges U(0.05,1) at lognormal(ln 1e-3, 2)
separation, 10% near-parallel, 5% intersecting), FP64 coordinates resident in HBM.
A step is one pass of the narrowphase over the 2^24 pairs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Ours: the headline method timed with CUDA events.  Default: the learned hybrid
(delta_pairs_run_learned: optional MLP warm start, FP32 projections, one FP64 feature,
FP64 separating-plane certificate at 1e-6, exact DELTA_BF_CERT for every uncertified pair)
in the configuration its autotuner times fastest (network on or off, projection sweeps);
the network-on and network-off arms, bf_cert and the plain FP64 bf kernel are timed beside
it on the same pairs.  `e2e` goes through the C ABI's host-buffer entry point
(delta_pairs_run_learned_host, or delta_pairs_run_host for a pair method) with pinned host
inputs, copies included.
Reference: the reference's own bfSolver (oracle/_ref, compiled from its sources) over a
bounded sample of the same pairs on all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "triangle-pair tests/sec and timesteps/sec at 1 B200: learned+FP32 vs plain FP64 at equal contacts"
BYTES_PER_PAIR = 144 + 56 + 1  # FP64 in (18 doubles) + out (P, Q, dist) + 1 flag byte
FLOPS_BF = 1214  # algorithmic FP ops of bfSolver per pair (747 add, 439 mul, 13 div, 15 sqrt)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--method", default="learned",
                    help="learned (the learned hybrid, configuration autotuned) or a pair method: bf_cert, bf, ...")
    ap.add_argument("--weights", default=None, help="warm-start checkpoint (default: the bundled one)")
    ap.add_argument("--learned-config", default="auto",
                    help="auto (autotuned) or network:sweeps:features, e.g. off:1:3, to pin the learned hybrid's "
                         "setting (no tuning, no comparison arms)")
    ap.add_argument("--pairs-log2", type=int, default=24)
    ap.add_argument("--passes", type=int, default=32,
                    help="passes over the resident pair batch per timed step (32 x 2^24 pairs: the timed region "
                         "of the default 20-step run lasts about a second, long enough for the clock record)")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--method-table", type=int, default=1,
                    help="1: time every pair method in FP64 and FP32 and state each result's error per class")
    ap.add_argument("--timestep-arms", default="",
                    help="comma-separated subset of the time-step arms to run (e.g. bf_cert_culled_graph under a "
                         "profiler); default all, with their comparisons")
    ap.add_argument("--min-timed-s", type=float, default=1.0,
                    help="a time-step arm whose steps take less runs again from the same initial state until its "
                         "timed total reaches this (0: one run, e.g. under a profiler)")
    ap.add_argument("--timestep-steps", type=int, default=1000,
                    help="time steps of the 256-icosphere lattice (its configuration's full length)")
    ap.add_argument("--hopper-steps", type=int, default=2000,
                    help="time steps of the 10,000-particle hopper (its configuration's full length)")
    ap.add_argument("--box-steps", type=int, default=-1,
                    help="time steps of the 200,000-particle box (default -1: its configuration's 500 on one GPU, "
                         "none on several, since every rank would build the 53 M-triangle scene)")
    return ap.parse_args()


def workload_config(n):
    return {
        "workload": "narrowphase microbenchmark: independent triangle pairs, lognormal(ln 1e-3, 2) separation, "
                    "10% near-parallel, 5% intersecting, FP64 coordinates",
        "pairs_per_gpu": n,
        "l2": "inputs larger than L2 (144 B/pair FP64 in HBM), no flush",
    }


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the sampler is running once its first line is in; samples before the timed
            # region starts are dropped
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 5.0:
                time.sleep(0.01)
            self.rows.clear()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peak_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


def profiled_traffic(kernel: str, n: int):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, scaled to n pairs."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        t = json.loads(p.read_text())[kernel]
        return float(t["dram_bytes_per_pair"]) * n
    except (KeyError, ValueError):
        return None


def profiled_flops(kernel: str):
    """(FP32, FP64) FLOP per pair of `kernel` counted by ncu (committed summary), or None."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        t = json.loads(p.read_text())[kernel]
        return float(t["fp32_flop_per_pair"]), float(t["fp64_flop_per_pair"]), t["flop_source"]
    except (KeyError, ValueError):
        return None


def cpu_reference_rate(a, b, sample: int, min_seconds: float):
    """The reference's bfSolver (oracle/_ref, or the oracle port when absent) over `sample`
    pairs on all host threads; repeated until min_seconds.  Returns (pairs/s, cores, kind)."""
    from oracle.oracle import Oracle, Reference

    cores = os.cpu_count() or 1
    if Reference.available("omp"):
        lib, kind = Reference("omp"), "reference"
    else:
        lib, kind = Oracle(), "port"
    a_s = np.ascontiguousarray(a[:, :sample]); b_s = np.ascontiguousarray(b[:, :sample])
    lib.pairs(0, a_s[:, :1024], b_s[:, :1024], nthreads=cores)  # warm-up
    done, t0 = 0, time.perf_counter()
    while True:
        lib.pairs(0, a_s, b_s, nthreads=cores, with_flags=False)
        done += sample
        el = time.perf_counter() - t0
        if el >= min_seconds:
            break
    return done / el, cores, kind


MIN_TIMED_S = 1.0  # the least timed total of a time-step arm (repeated runs of the same steps); --min-timed-s


def _time_sim(ctx, stream, sim, steps, params, graph):
    import torch

    c0 = sim.counters()
    l0 = ctx.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    sim.step(steps, params, graph=graph)
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    # graph replays run on the simulation's own stream: the wall clock brackets them
    t = wall if graph else e0.elapsed_time(e1) / 1e3
    c1 = sim.counters()
    tri = c1["triangle_pairs"] - c0["triangle_pairs"]
    solved = c1["solved"] - c0["solved"]
    return {"steps_per_s": steps / t, "ms_per_step": 1e3 * t / steps, "triangle_pair_tests_per_s": tri / t,
            "solved_pairs_per_s": solved / t,
            "triangle_pairs_per_step": tri / steps, "solved_pairs_per_step": (c1["solved"] - c0["solved"]) / steps,
            "body_pairs_per_step": (c1["body_pairs"] - c0["body_pairs"]) / steps,
            "gpu_launches": ctx.launches - l0, "timer": "wall clock around synchronised replays" if graph else
            "CUDA events"}


def cpu_timestep_rate(scene, params, steps: int):
    """Timesteps/s of the reference-driven time step (oracle/_ref, ref_sim.cpp: the reference's
    bf() on every triangle pair of every candidate body pair, getContactsForces,
    updateAngular, updateRotationMatrix, updateVertices) on all host threads."""
    from oracle.oracle import Reference

    if not Reference.available("omp"):
        return None
    ref = Reference("omp")
    dt = float(params.dt)
    g = [float(params.gravity[k]) for k in range(3)]
    warm, _ = ref.simulate(scene, dt, g, 1)  # the first detection (contacts for the next step)
    t0 = time.perf_counter()
    _, cps = ref.simulate(warm, dt, g, steps)
    el = time.perf_counter() - t0
    return {"value": steps / el, "unit": "timesteps/s", "cores": os.cpu_count() or 1, "kind": "reference",
            "sample": f"{steps} time steps after one warm-up step; the reference's bf() over all triangle pairs "
                      "of the candidate body pairs, getContactsForces with forces.cpp's compiled constants, "
                      "dynamics.cpp's updates; OpenMP over candidate pairs and bodies",
            "contacts_last_step": int(cps[-1]) if len(cps) else 0}


def timestep_section(ctx, stream, scene, workload, steps: int, warmup: int, params, cpu_steps: int = 0,
                     arm_filter=None):
    """Timesteps/s of a scene with the plain FP64 bf driver (every triangle pair of every
    candidate body pair, as the reference) and with the certified FP32 driver (exact box
    culling + bf_cert), stepped and replayed as a CUDA graph.  All three must give the same
    trajectory bit for bit."""
    from delta_b200.detection import DRV_BF, DRV_BF_CERT, DRV_BF_CULLED, DRV_LEARNED
    from delta_b200.engine import Simulation

    out, states = {}, {}
    arms = [("fp64_bf", DRV_BF, False, steps), ("fp64_bf_culled", DRV_BF_CULLED, False, steps),
            ("fp64_bf_culled_graph", DRV_BF_CULLED, True, steps), ("bf_cert_culled", DRV_BF_CERT, False, steps),
            ("bf_cert_culled_graph", DRV_BF_CERT, True, steps), ("learned_culled_graph", DRV_LEARNED, True, steps)]
    def timed_arm(c, drv, graph, k, tune=False):
        """Times k steps after the warm-up; an arm whose timed steps take under
        MIN_TIMED_S runs again from the same initial state (a fresh simulation) until the
        timed total reaches it.  Returns (result of the totals, state after the first run)."""
        total_t, total_steps, first, state, reps, shape = 0.0, 0, None, None, 0, None
        while True:
            sim = Simulation(c, scene, drv)
            if tune and reps == 0:
                # the certified driver after delta_sim_autotune (the shapes are the
                # context's, so later repeats use them), with the same steps before the
                # timed region as the other arms
                if warmup > 1:
                    sim.step(warmup - 1, params, graph=graph)
                shape = sim.autotune(reps=3)
                sim.step(1, params, graph=graph)  # records the graph with the chosen shapes
            else:
                sim.step(warmup, params, graph=graph)
            r = _time_sim(c, stream, sim, k, params, graph)
            if reps == 0:
                first, state = r, sim.state()
                if graph:  # the graph step's skin list: its capacity and the builds inside the replays
                    first = dict(first, skin_list=sim.skin_stats())
            sim.close()
            total_t += k / r["steps_per_s"]
            total_steps += k
            reps += 1
            if total_t >= MIN_TIMED_S or reps >= 64:
                break
        sps = total_steps / total_t
        res = dict(first, steps_per_s=sps, ms_per_step=1e3 / sps,
                   triangle_pair_tests_per_s=first["triangle_pairs_per_step"] * sps,
                   solved_pairs_per_s=first["solved_pairs_per_step"] * sps, repeats=reps,
                   timed_seconds=total_t)
        if shape is not None:
            res["launch_shape"] = shape
        return res, state

    only = set(arm_filter) if arm_filter else None
    for name, drv, graph, k in arms:
        if only is None or name in only:
            out[name], states[name] = timed_arm(ctx, drv, graph, k)
    if only is None or "bf_cert_culled_graph_tuned" in only:
        from delta_b200.narrowphase import Context

        tctx = Context(0, stream=stream.cuda_stream)
        try:
            out["bf_cert_culled_graph_tuned"], states["bf_cert_culled_graph_tuned"] = timed_arm(
                tctx, DRV_BF_CERT, True, steps, tune=True)
        finally:
            tctx.close()
    res = {"workload": workload, "steps": steps, "warmup": warmup, **out}
    if only is not None:  # a subset of the arms (e.g. under a profiler): no comparisons
        return res
    ref = states["fp64_bf"]
    exact = [n for n in states if n != "learned_culled_graph"]
    same = all(np.array_equal(ref[k], states[n][k]) for n in exact for k in ("pos", "vel", "rot", "x"))
    lrn = states["learned_culled_graph"]
    out["learned_culled_graph"]["vs_fp64_bf"] = {
        "max_abs_pos_m": float(np.max(np.abs(lrn["pos"] - ref["pos"]))),
        "max_abs_vel_m_per_s": float(np.max(np.abs(lrn["vel"] - ref["vel"]))),
        "bit_identical": bool(all(np.array_equal(ref[k], lrn[k]) for k in ("pos", "vel", "rot", "x")))}
    sps = {k: v["steps_per_s"] for k, v in out.items()}
    cpu = cpu_timestep_rate(scene, params, cpu_steps) if cpu_steps > 0 else None
    return {**res, "cpu_baseline": cpu,
            "speedup": sps["bf_cert_culled_graph"] / sps["fp64_bf"],
            "speedup_learned": sps["learned_culled_graph"] / sps["fp64_bf"],
            "speedup_tuned": sps["bf_cert_culled_graph_tuned"] / sps["fp64_bf"],
            "speedup_from_culling": sps["fp64_bf_culled"] / sps["fp64_bf"],
            "speedup_from_precision": sps["bf_cert_culled_graph"] / sps["fp64_bf_culled_graph"],
            "speedup_note": "culling: culled FP64 bf vs plain FP64 bf (both stepped); precision: certified "
                            "FP32+FP64 vs FP64 bfSolver on the same survivors (both graph-replayed)",
            "trajectories_bit_identical": bool(same),
            "bit_identical_arms": exact}


def run_reference(args, rank, world):
    n = 1 << args.pairs_log2
    if rank != 0:
        return
    from delta_b200.scenarios import narrowphase_pairs_chunked

    sample = min(n, 1 << 22)
    a, b, _, _ = narrowphase_pairs_chunked(sample, seed=args.seed)
    from oracle.oracle import Oracle, Reference

    cores = os.cpu_count() or 1
    lib, kind = (Reference("omp"), "reference") if Reference.available("omp") else (Oracle(), "port")
    for _ in range(args.warmup):
        lib.pairs(0, a, b, nthreads=cores, with_flags=False)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        lib.pairs(0, a, b, nthreads=cores, with_flags=False)
    el = time.perf_counter() - t0
    rate = sample * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {**workload_config(n), "method": "reference bfSolver (FP64, CPU)"},
        "cpu_baseline": {"value": rate, "unit": "pairs/s", "cores": cores, "kind": kind,
                         "sample": f"{sample} pairs of the workload per step, bfSolver FP64 on {cores} threads"},
        "e2e": {"value": rate, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    global MIN_TIMED_S
    args = parse()
    MIN_TIMED_S = args.min_timed_s
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.box_steps < 0:
        args.box_steps = 500 if world == 1 else 0
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    n = 1 << args.pairs_log2
    # host-side generation first (spawned pool, before any CUDA initialisation)
    from delta_b200.scenarios import narrowphase_pairs_chunked

    a_np, b_np, _, cls_np = narrowphase_pairs_chunked(n, seed=args.seed + 7919 * rank)

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from delta_b200.narrowphase import METHODS, Context, autotune, pairs_device, pairs_host

    stream = torch.cuda.current_stream()
    ctx = Context(local, stream.cuda_stream)
    a = torch.from_numpy(a_np).cuda()
    b = torch.from_numpy(b_np).cuda()

    def new_out():
        return (torch.empty((3, n), dtype=torch.float64, device="cuda"),
                torch.empty((3, n), dtype=torch.float64, device="cuda"),
                torch.empty(n, dtype=torch.float64, device="cuda"), torch.empty(n, dtype=torch.uint8, device="cuda"))

    out, out64 = new_out(), new_out()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(run, outs, steps, warmup):
        for _ in range(warmup):
            run(outs)
        barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        l0 = ctx.launches
        ev[0].record(stream)
        for i in range(steps):
            run(outs)
            ev[i + 1].record(stream)
        barrier()
        per = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
        return ev[0].elapsed_time(ev[steps]), per, ctx.launches - l0

    def max_ranks(vals):
        t = torch.tensor(vals, dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return t.tolist()

    def pair_run(m):
        return lambda outs: pairs_device(ctx, m, a, b, out=outs)

    def per_step(run):
        """One timed step: args.passes passes of `run` over the resident batch."""
        def step(outs):
            for _ in range(args.passes):
                run(outs)
        return step

    # launch shapes of the pair kernels chosen by the autotuner on this rank's pairs
    tuned = {"bf_cert": autotune(ctx, METHODS["bf_cert"], a, b, out=out),
             "bf": autotune(ctx, METHODS["bf"], a, b, out=out64)}
    learned_info = None
    if args.method == "learned":
        from delta_b200.learned import WarmStartMLP, default_weights, learned_pairs, learned_pairs_host, refine, tune

        model = WarmStartMLP.load(ctx, args.weights)
        if args.learned_config == "auto":
            tuning = tune(ctx, model, a, b)
            best = tuning[0]
        else:
            net_s, sw_s, f_s = args.learned_config.split(":")
            best = {"network": net_s == "on", "sweeps": int(sw_s), "features": int(f_s),
                    "certified_fraction": None}
            tuning = [best]
        use_model = model if best["network"] else None
        sweeps, feats = best["sweeps"], best["features"]

        def headline(outs):
            return learned_pairs(ctx, use_model, a, b, sweeps, out=outs, features=feats)
    else:
        headline = pair_run(METHODS[args.method])

    peak, peak_kind = measured_peak_hbm()
    with ClockSampler(local) as clk:
        total_ms, per_ms, launches = timed(per_step(headline), out, args.steps, args.warmup)
    # the plain FP64 bf kernel on the same pairs (comparison arm, not the headline)
    steps64 = max(3, args.steps // 2)
    total64_ms, per64_ms, _ = timed(pair_run(METHODS["bf"]), out64, steps64, 2)
    total_ms, total64_ms = max_ranks([total_ms, total64_ms])
    value = world * n * args.passes * args.steps / (total_ms / 1e3)
    value64 = world * n * steps64 / (total64_ms / 1e3)

    # parity of the headline against plain FP64 bf on this rank's pairs
    torch.cuda.synchronize()
    d, d64 = out[2], out64[2]
    fin = torch.isfinite(d64)
    rel = ((d - d64).abs() / d64.clamp_min(1e-300))[fin].max().item()
    same = ((out[0] == out64[0]).all(0) & (out[1] == out64[1]).all(0) & ((d == d64) | (d.isnan() & d64.isnan())))
    contacts = {}
    for thr in (1e-4, 1e-3, 1e-2):
        outside = (d64 - thr).abs() > 1e-6 * thr
        contacts[f"{thr:g}"] = {"fp64_contacts": int((d64 <= thr).sum().item()),
                                "mismatches_outside_band": int((((d <= thr) != (d64 <= thr)) & outside).sum().item()),
                                "pairs_in_band": int((~outside).sum().item())}
    parity = {"pairs_bit_identical_fraction": same.double().mean().item(), "max_rel_dist_err": rel,
              "rel_tol": 1e-6 if args.method == "learned" else 0.0,
              "contact_sets_at_threshold": contacts,
              "band": "|d_fp64 - threshold| <= 1e-6 threshold"}

    if args.method == "learned":
        # comparison arms on the same pairs and the same timing protocol
        arms = {}
        best_on = next((r for r in tuning if r["network"]), None)
        best_off = next((r for r in tuning if not r["network"]), None)
        k = max(3, args.steps // 2)
        arm_out = new_out()
        arm_runs = [("bf_cert", pair_run(METHODS["bf_cert"]), None)]
        if args.learned_config == "auto":
            arm_runs += [
                ("learned_network_on", lambda o: learned_pairs(ctx, model, a, b, best_on["sweeps"], out=o,
                                                               features=best_on["features"]), best_on),
                ("learned_network_off", lambda o: learned_pairs(ctx, None, a, b, best_off["sweeps"], out=o,
                                                                features=best_off["features"]), best_off)]
        for name, run, r in arm_runs:
            t_ms, _, _ = timed(run, arm_out, k, 2)
            (t_ms,) = max_ranks([t_ms])
            arms[name] = {"value": world * n * k / (t_ms / 1e3), "unit": "pairs/s", "ms_per_step": t_ms / k}
            if r is not None:
                arms[name].update(sweeps=r["sweeps"], features=r["features"],
                                  certified_fraction=r["certified_fraction"])
        # per-kernel breakdown of the headline configuration
        x0 = model.predict(a, b) if use_model is not None else None
        ref_out = new_out()

        def ev_time(fn, reps=max(3, args.steps // 2)):
            fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1) / reps

        refine_ms = ev_time(lambda: refine(ctx, a, b, x0, sweeps, out=ref_out, features=feats))
        infer_ms = ev_time(lambda: model.predict(a, b, out=x0)) if use_model is not None else 0.0
        head_ms = total_ms / (args.steps * args.passes)
        ckpt = json.loads(default_weights().with_suffix(".json").read_text()) if args.weights is None else None
        learned_info = {
            "config": {"network": bool(best["network"]), "sweeps": sweeps, "features": feats,
                       "certified_fraction": best["certified_fraction"],
                       "chosen_by": "delta_b200.learned.tune: CUDA-event timing of every (network, sweeps, features)"},
            "tuning": tuning,
            "arms": arms,
            "breakdown_ms": {"mlp_inference": infer_ms, "refine_and_certify": refine_ms,
                             "exact_fallback_and_list": max(head_ms - refine_ms - infer_ms, 0.0)},
            "network_gain_certified_fraction": {
                f"sweeps{r['sweeps']}_features{r['features']}": {
                    "network": r["certified_fraction"],
                    "plain": next((x["certified_fraction"] for x in tuning if not x["network"] and
                                   x["sweeps"] == r["sweeps"] and x["features"] == r["features"]), None)}
                for r in tuning if r["network"]},
            "checkpoint": None if ckpt is None else {
                "training_pairs": ckpt["training_pairs"], "epochs": ckpt["epochs"], "batch": ckpt["batch"],
                "lr": ckpt["lr"], "train_samples_per_second": ckpt["train_samples_per_second"],
                "eval_loss": ckpt["evaluation"]["loss"], "device": ckpt["device"]},
        }

    # the method x precision table of the microbenchmark: every pair method in FP64 and FP32
    # on the same pairs, throughput (CUDA events) and the error of each result per class
    methods_table = None
    if args.method_table:
        from delta_b200.scenarios import CLASS_NAMES

        cls = torch.from_numpy(cls_np).cuda()
        d_bf = out64[2].clone()
        tab_out = new_out()
        methods_table = {}
        for mname in ("bf", "penalty", "penalty_iter", "gjk", "hybrid"):
            row = {}
            d_prec = {}
            for prec, pname in ((0, "f64"), (1, "f32")):
                def run(o, m=METHODS[mname], pr=prec):
                    pairs_device(ctx, m, a, b, precision=pr, max_error=1e-3, out=o)
                t_ms, _, _ = timed(run, tab_out, 3, 1)
                (t_ms,) = max_ranks([t_ms])
                d_prec[pname] = tab_out[2].clone()
                row[pname] = {"value": world * n * 3 / (t_ms / 1e3), "unit": "pairs/s", "ms_per_step": t_ms / 3}

            def err_stats(x, ref):
                per = {}
                for c, cname in enumerate(CLASS_NAMES):
                    sel = (cls == c) & torch.isfinite(ref) & (ref > 0)
                    e = (x[sel] - ref[sel]).abs()
                    r = (e / ref[sel]).double()
                    fin = torch.isfinite(r)
                    r, ea = r[fin], e[fin]
                    per[cname] = {"pairs": int(sel.sum().item()),
                                  "nonfinite": int((~fin).sum().item()),
                                  "rel_p50": float(torch.quantile(r[:1 << 24].float(), 0.5).item()) if r.numel() else None,
                                  "rel_p99": float(torch.quantile(r[:1 << 24].float(), 0.99).item()) if r.numel() else None,
                                  "rel_max": float(r.max().item()) if r.numel() else None,
                                  "abs_max": float(ea.max().item()) if ea.numel() else None}
                return per
            row["f32_vs_f64_same_method"] = err_stats(d_prec["f32"], d_prec["f64"])
            row["f64_vs_fp64_bf"] = err_stats(d_prec["f64"], d_bf)
            row["f32_vs_fp64_bf"] = err_stats(d_prec["f32"], d_bf)
            methods_table[mname] = row
        del tab_out, d_prec, d_bf

    # end to end through the C ABI with pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        ha = torch.from_numpy(a_np).pin_memory().numpy()
        hb = torch.from_numpy(b_np).pin_memory().numpy()
        hp = torch.empty((3, n), dtype=torch.float64).pin_memory().numpy()
        hq = torch.empty((3, n), dtype=torch.float64).pin_memory().numpy()
        hd = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
        hf = torch.empty(n, dtype=torch.uint8).pin_memory().numpy()
        if args.method == "learned":
            def host_run():
                learned_pairs_host(ctx, use_model, ha, hb, sweeps, out=(hp, hq, hd, hf), features=feats)
            path = "delta_pairs_run_learned_host (C ABI), pinned host buffers, copies in the timed region"
        else:
            def host_run():
                pairs_host(ctx, METHODS[args.method], ha, hb, out=(hp, hq, hd, hf))
            path = "delta_pairs_run_host (C ABI), pinned host buffers, copies in the timed region"
        host_run()  # warm-up (allocates scratch)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            host_run()
        barrier()
        (el,) = max_ranks([time.perf_counter() - t0])
        # the PCIe bound: a plain pinned host-to-device copy of the A planes, after the run
        dev_a = torch.empty(ha.shape, dtype=torch.float64, device="cuda")
        src_a = torch.from_numpy(ha)
        for _ in range(2):
            dev_a.copy_(src_a, non_blocking=True)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(3):
            dev_a.copy_(src_a, non_blocking=True)
        torch.cuda.synchronize()
        h2d_gbs = 3 * ha.nbytes / (time.perf_counter() - t1) / 1e9
        del dev_a
        e2e = {"value": world * n * args.e2e_steps / el, "unit": "pairs/s",
               "h2d_bytes_per_step": int(ha.nbytes + hb.nbytes),
               "d2h_bytes_per_step": int(hp.nbytes + hq.nbytes + hd.nbytes + hf.nbytes), "path": path,
               "pinned_h2d_gbs": h2d_gbs,
               "h2d_bound_pairs_per_s": world * h2d_gbs * 1e9 / ((ha.nbytes + hb.nbytes) / n)}

    ts = hop = box = None
    arm_filter = [a for a in args.timestep_arms.split(",") if a]
    if args.timestep_steps > 0:
        from delta_b200.engine import StepParams
        from delta_b200.scenarios import hopper_scene, lattice_scene

        ts = timestep_section(
            ctx, stream, lattice_scene(args.seed),
            "256 perturbed icospheres (80 tri) on a 8x4x8 lattice over a 2-triangle floor, FP64, dt 1e-5, k 1e6, "
            "damping 0.1", args.timestep_steps, 3,
            StepParams.make(dt=1e-5, gravity=(0.0, -9.81, 0.0), spring=1e6, damper=0.1, friction=0.0),
            cpu_steps=3 if (rank == 0 and world == 1 and not args.no_cpu_baseline) else 0, arm_filter=arm_filter)
        if args.box_steps > 0:
            from delta_b200.scenarios import box_scene

            box = timestep_section(
                ctx, stream, box_scene(200000, seed=args.seed),
                "200,000 perturbed spheres of {80,160,320,500} triangles (r 4-12 mm, 53 M triangles) poured from a "
                "lattice into a 0.6 x 1.2 x 0.6 m box of 12 wall triangles, FP64, dt 2e-6", args.box_steps, 2,
                StepParams.make(dt=2e-6, gravity=(0.0, -9.81, 0.0), spring=1e6, damper=0.1, friction=0.0),
                arm_filter=arm_filter)
        if args.hopper_steps > 0:
            hop = timestep_section(
                ctx, stream, hopper_scene(10000, seed=args.seed),
                "10,000 perturbed spheres of {40,80,160,320} triangles (r 5-15 mm) over a conical hopper of 2,048 "
                "wall triangles (30 deg, 8 cm outlet), FP64, dt 5e-6", args.hopper_steps, 3,
                StepParams.make(dt=5e-6, gravity=(0.0, -9.81, 0.0), spring=1e6, damper=0.1, friction=0.0),
                cpu_steps=2 if (rank == 0 and world == 1 and not args.no_cpu_baseline) else 0, arm_filter=arm_filter)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, kind = cpu_reference_rate(a_np, b_np, sample=min(n, 1 << 22), min_seconds=10.0)
        cpu = {"value": rate, "unit": "pairs/s", "cores": cores, "kind": kind,
               "sample": f"{min(n, 1 << 22)} pairs of the workload, reference bfSolver FP64, repeated >= 10 s"}

    if rank == 0:
        if args.method == "learned":
            # dominant kernel of the headline: the refine/certify kernel (or the MLP when on)
            kname = "k_learned_refine"
            bpp = BYTES_PER_PAIR + (16 if use_model is not None else 0)
            kern_ms = learned_info["breakdown_ms"]["refine_and_certify"]
            traffic = profiled_traffic("learned_refine", n)
        else:
            kname = f"k_pairs<{args.method}>"
            bpp = BYTES_PER_PAIR
            kern_ms = float(np.mean(per_ms)) / args.passes
            traffic = profiled_traffic(args.method, n)
        achieved = bpp * n / (kern_ms / 1e3) / 1e9
        # compute side: FP32/FP64 operations per pair (ncu counts of the same kernel) at the
        # measured rate, against CUDA-core peaks derived from 148 SMs x max SM clock x lanes
        # x 2 (FMA): 128 FP32 and 64 FP64 lanes per SM
        compute = None
        fl = profiled_flops("learned_refine") if args.method == "learned" else None
        if fl is not None:
            clk_ghz = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text()).get("sm_max_mhz", 1965.0)) / 1e3 \
                if (ROOT / "MEASURED_PEAKS.json").exists() else 1.965
            rate = n / (kern_ms / 1e3)
            p32, p64 = 148 * clk_ghz * 128 * 2 / 1e3, 148 * clk_ghz * 64 * 2 / 1e3
            compute = {"fp32_flop_per_pair": fl[0], "fp64_flop_per_pair": fl[1], "source": fl[2],
                       "fp32_tflops": fl[0] * rate / 1e12, "fp32_peak_tflops_derived": p32,
                       "fp32_frac": fl[0] * rate / 1e12 / p32,
                       "fp64_tflops": fl[1] * rate / 1e12, "fp64_peak_tflops_derived": p64,
                       "fp64_frac": fl[1] * rate / 1e12 / p64,
                       "note": "issue-bound: ~76% of scheduler cycles issue (ncu); the FP pipes are not the limit"}
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {**workload_config(n), "method": args.method, "passes_per_step": args.passes,
                       "step": f"{args.passes} passes of the narrowphase over the resident {n}-pair batch",
                       "comparison": "plain FP64 bf kernel on the same pairs"},
            "fp64_bf": {"value": value64, "unit": "pairs/s", "ms_per_step": total64_ms / steps64},
            "autotuned_launch": tuned,
            "speedup_vs_fp64_bf": value / value64,
            "parity_vs_fp64_bf": parity,
            "learned": learned_info,
            "roofline": {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": bpp * n, "kernel_ms": kern_ms, "compute": compute},
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "e2e": e2e,
            "methods_fp64_fp32": methods_table,
            "cpu_baseline": cpu,
            "timestep": ts,
            "timestep_hopper": hop,
            "timestep_box": box,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
