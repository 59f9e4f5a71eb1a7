#!/usr/bin/env python
"""Benchmark of the FDTD step (Gcell-steps/s and fraction of the HBM roofline).

Workload: the single large solve, 256^3 cells, h = 2.5 mm, 16-cell PML, three
static rigid bodies (sphere, box, ellipsoid) with a Gaussian-in-time boundary
acceleration of 1e3 m/s^2, 64 listeners; seeded synthetic scene.  One bench
"step" is one FDTD time step of that solve (every cell updated once, listeners
sampled).  Headline precision: FP32 with compensated accumulation; the FP64
fused path, the plain FP64 path (one kernel per reference phase) and the FP32
listener error against FP64 are reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own independent solve on its own GPU (the
path shards across solves, not within one): value = sum over ranks of cells x
steps / max-over-ranks time, scaling "weak".
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-steps/s & %HBM roofline; served solves/s, p99, at ≤1e-4 rel-L2 vs FP64"
UNIT = "Gcell-steps/s"
L2_BYTES = 126 * 2**20


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def bench_scene(steps_for_accuracy=None):
    from acoustics_b200.scene import config2
    return config2()


def cpu_baseline(scene, budget_s: float, max_steps: int):
    """The FP64 CPU oracle (restatement of the reference step) on the host cores."""
    from oracle import loader
    threads = loader.set_threads(os.cpu_count() or 1)
    o = loader.OracleSolver(scene)
    o.step(1)  # warm-up, untimed
    t0 = time.perf_counter()
    n = 0
    while n < max_steps:
        o.step(1)
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    o.close()
    return scene.n_cells * n / dt / 1e9, n, threads, dt


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    sc = bench_scene()
    budget = float(os.environ.get("FDTD_REF_BUDGET_S", "120"))
    val, n, threads, dt = cpu_baseline(sc, budget, max(1, args.steps))
    sample = (f"{n} full FDTD steps of the 256^3 solve ({sc.n_cells} cells) after 1 warm-up step, "
              f"{dt:.1f} s, FP64 CPU oracle (restatement of the reference step; the reference itself "
              f"cannot be built here)")
    line = {
        "metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": n, "warmup": 1, "ms_per_step": dt / n * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": sc.name, "cells": sc.n_cells, "divisions": list(sc.divisions),
                   "pml_width": sc.pml_width, "listeners": sc.n_listeners, "objects": len(sc.objects)},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def read_traffic(precision: str, n: int):
    """DRAM bytes per step of the step-kernel group from the committed ncu summary
    (profiles/kernel_traffic.txt: `precision cells bytes` per line)."""
    p = os.path.join(ROOT, "profiles", "kernel_traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 3 and not line.startswith("#") and parts[0] == precision and int(parts[1]) == n:
                return float(parts[2])
    return None


def profile_run(args):
    """Create the bench solve and run a few steps, nothing else: the command the
    committed ncu summaries under profiles/ were captured with."""
    from acoustics_b200 import scene as S
    from acoustics_b200.solver import PML_WaveSolver
    prec = S.PRECISION_FP32_COMPENSATED if args.precision == "fp32" else S.PRECISION_FP64
    if args.profile_batch:
        # the 64 uneven scenes stepped eagerly (no graphs), so every kernel is listed
        from acoustics_b200.batch import SolveBatch
        scenes = S.config3()
        b = SolveBatch(scenes, precision=prec, graph_steps=0, tile_y=args.tile_y, x_chunk=args.x_chunk, tune=False)
        b.step(args.steps)
        launches = b.last_launch_count()
        b.close()
        print(json.dumps({"profile_run": "config3_batch", "members": len(scenes), "steps": args.steps,
                          "launches": launches}))
        return 0
    if args.profile_moving:
        # configuration 5: every step reclassifies the two moving spheres
        sc = S.config5()
        g = PML_WaveSolver(sc, precision=prec)
        y = g.step(3 + args.steps)
        g.close()
        print(json.dumps({"profile_run": sc.name, "cells": sc.n_cells, "steps": 3 + args.steps,
                          "max_abs_listener": float(np.abs(y).max())}))
        return 0
    sc = S.config2(n=args.profile_n)
    kern = S.KERNEL_PHASED if args.precision == "fp64-plain" else S.KERNEL_FUSED
    g = PML_WaveSolver(sc, precision=prec, kernel=kern, tile_y=args.tile_y, x_chunk=args.x_chunk,
                       shell_staging=args.profile_staging)
    y = g.step(3 + args.steps)
    g.close()
    print(json.dumps({"profile_run": sc.name, "cells": sc.n_cells, "steps": 3 + args.steps,
                      "max_abs_listener": float(np.abs(y).max())}))
    return 0


def bench_batched(peak: float, fp64_check: bool = True):
    """64 uneven scenes (grid edges log-uniform in [48, 160], 1000-3000 steps, 1-3
    bodies) stepped as one batch, FP32 compensated, against the same scenes run one
    by one through PML_WaveSolver.  Cell-steps count every step after the first
    (classifying) one, which fdtd_batch_add runs per member before the timed loop."""
    import torch

    from acoustics_b200 import scene as S
    from acoustics_b200.batch import SolveBatch, scene_info
    from acoustics_b200.solver import PML_WaveSolver
    scenes = S.config3()
    P32 = S.PRECISION_FP32_COMPENSATED
    infos = [scene_info(sc, precision=P32) for sc in scenes]
    cell_steps = sum(i.n_cells * (sc.steps - 1) for i, sc in zip(infos, scenes))
    alg = sum(i.algorithmic_bytes_per_step * (sc.steps - 1) for i, sc in zip(infos, scenes))
    out = {"workload": "config3: 64 uneven scenes, edges log-uniform [48,160], 1000-3000 steps",
           "scenes": len(scenes), "cells": int(sum(i.n_cells for i in infos)),
           "cell_steps": int(cell_steps), "graph_steps": 16}
    # tile shapes from the autotuner (every candidate timed on a sample of the
    # scenes, outside the timed region; cached per grid class)
    from acoustics_b200 import autotune
    t0 = time.perf_counter()
    tuned = autotune.tune(scenes, P32)
    out["autotune"] = {"x_chunk": tuned["x_chunk"], "tile_y": tuned["tile_y"], "key": tuned["key"],
                       "timings_ms_per_step": tuned["timings_ms"], "sample_scenes": tuned["sample_scenes"],
                       "seconds": time.perf_counter() - t0}
    b = SolveBatch(scenes, precision=P32, graph_steps=16, x_chunk=tuned["x_chunk"], tile_y=tuned["tile_y"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.run()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    y32 = [b.output(m) for m in range(len(scenes))]
    b.close()
    out.update({"seconds": dt, "gcell_steps_s": cell_steps / dt / 1e9,
                "achieved_gbs": alg / dt / 1e9, "hbm_frac": alg / dt / 1e9 / peak})
    # one by one, same scenes and options, stepping only (creation outside)
    solvers = [PML_WaveSolver(sc, precision=P32, graph_steps=16) for sc in scenes]
    for g in solvers:
        g.step(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for g, sc in zip(solvers, scenes):
        g.step(sc.steps - 1)
    torch.cuda.synchronize()
    dt1 = time.perf_counter() - t0
    for g in solvers:
        g.close()
    out.update({"one_by_one_seconds": dt1, "one_by_one_gcell_steps_s": cell_steps / dt1 / 1e9,
                "speedup_vs_one_by_one": dt1 / dt})
    if fp64_check:
        b64 = SolveBatch(scenes, precision=S.PRECISION_FP64, graph_steps=16, tune=False)
        b64.run()
        y64 = [b64.output(m) for m in range(len(scenes))]
        b64.close()
        errs = [float(np.linalg.norm(a - c) / np.linalg.norm(c)) for a, c in zip(y32, y64)]
        out["listener_rel_l2_vs_fp64_max"] = max(errs)
        out["listener_rel_l2_vs_fp64_median"] = float(np.median(errs))
    return out


def bench_moving(peak: float):
    """Configuration 5: 384x384x256, two ballistic spheres that touch mid-run,
    every step reclassified (solid / ghost cells, fresh-cell MLS); the whole
    6000-step run from creation, FP32 compensated and FP64, CUDA-event time on
    the solver stream.  The FP32 listener series is checked against FP64."""
    import torch

    from acoustics_b200 import scene as S
    from acoustics_b200.solver import PML_WaveSolver
    sc = S.config5()
    out = {"workload": "config5: 384x384x256 moving spheres, per-step reclassification", "cells": sc.n_cells,
           "steps": sc.steps}
    ys = {}
    for name, prec in (("fp32", S.PRECISION_FP32_COMPENSATED), ("fp64", S.PRECISION_FP64)):
        g = PML_WaveSolver(sc, precision=prec)
        g.synchronize()
        ext = torch.cuda.ExternalStream(g.stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(ext)
        ys[name] = g.step(sc.steps)
        b.record(ext)
        b.synchronize()
        ms = a.elapsed_time(b) / sc.steps
        alg = float(g.info().algorithmic_bytes_per_step)
        out[name] = {"ms_per_step": ms, "gcell_steps_s": sc.n_cells / (ms / 1e3) / 1e9,
                     "hbm_frac": alg / (ms / 1e3) / 1e9 / peak, "overlapped_steps": g.overlapped_steps()}
        g.close()
    out["fp32_listener_rel_l2_vs_fp64"] = float(np.linalg.norm(ys["fp32"] - ys["fp64"]) / np.linalg.norm(ys["fp64"]))
    return out


def bench_served(peak: float, rate: float, n_requests: int, fifo_plain: bool = False):
    """Poisson request stream (config4) into the solve server (FP32, continuous
    batching) and, as the baseline, the same requests served first-in first-out
    one at a time by the plain FP64 GPU single-solve path (fused kernels, graphs);
    optionally also by the phased FP64 path (one kernel per reference phase)."""
    from acoustics_b200 import scene as S
    from acoustics_b200.batch import scene_info
    from acoustics_b200.server import SolveServer
    from acoustics_b200.solver import PML_WaveSolver
    reqs = S.config4(n_requests=n_requests, rate_per_s=rate)
    P32 = S.PRECISION_FP32_COMPENSATED
    infos = [scene_info(sc, precision=P32) for _, sc in reqs]
    cell_steps = sum(i.n_cells * sc.steps for i, (_, sc) in zip(infos, reqs))
    alg = sum(i.algorithmic_bytes_per_step * sc.steps for i, (_, sc) in zip(infos, reqs))
    out = {"workload": f"config4: {n_requests} Poisson arrivals at {rate}/s, edges log-uniform [64,256], "
                       f"1000-8000 steps, 16 listeners", "requests": n_requests, "cell_steps": int(cell_steps)}

    def serve(scale):
        # the same requests arriving `scale` times faster (seeded gaps / scale)
        with SolveServer(precision=P32, graph_steps=16, chunk_steps=32, tune_for=[sc for _, sc in reqs]) as srv:
            t0 = time.perf_counter()
            ids = []
            for t_arr, sc in reqs:
                d = t0 + t_arr / scale - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                ids.append(srv.submit(sc))
            lat = [srv.result(i)[1] for i in ids]
            st = srv.stats()
        return {"rate_per_s": rate * scale, "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)), "solves_per_s": st["solves_per_s"],
                "gcell_steps_s": st["cell_steps_per_s"] / 1e9,
                "hbm_frac": alg / st["span_s"] / 1e9 / peak if st["span_s"] > 0 else None,
                "span_s": st["span_s"], "peak_members": st["peak_members"],
                "peak_device_gb": st["peak_device_bytes"] / 1e9}

    def fifo(kernel, graph_steps):
        t0 = time.perf_counter()
        lat64 = []
        for t_arr, sc in reqs:
            d = t0 + t_arr - time.perf_counter()
            if d > 0:
                time.sleep(d)
            g = PML_WaveSolver(sc, precision=S.PRECISION_FP64, kernel=kernel, graph_steps=graph_steps)
            g.step(sc.steps)
            g.close()
            lat64.append(time.perf_counter() - (t0 + t_arr))
        span = time.perf_counter() - (t0 + reqs[0][0])
        return {"p50_latency_s": float(np.percentile(lat64, 50)), "p99_latency_s": float(np.percentile(lat64, 99)),
                "solves_per_s": n_requests / span, "gcell_steps_s": cell_steps / span / 1e9}

    # one untimed pass at the highest rate first: module loading, tile tuning and
    # the device blocks of the first members are not part of serving
    serve(16.0)
    base = serve(1.0)
    base.pop("rate_per_s")
    out.update(base)
    # faster arrivals until the GPU, not the stream, sets the pace
    out["rate_sweep"] = [serve(f) for f in (4.0, 16.0)]
    out["fifo_fp64_fused"] = fifo(S.KERNEL_FUSED, 16)
    out["solves_per_s_vs_fifo_fp64_fused"] = out["solves_per_s"] / out["fifo_fp64_fused"]["solves_per_s"]
    out["p99_vs_fifo_fp64_fused"] = out["p99_latency_s"] / out["fifo_fp64_fused"]["p99_latency_s"]
    if fifo_plain:
        out["fifo_fp64_plain"] = fifo(S.KERNEL_PHASED, 0)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64", "fp64-plain"])
    ap.add_argument("--graph-steps", type=int, default=16,
                    help="steps per CUDA graph (16; a timed run of 18-64 steps, even, uses one graph of its length)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--fifo-plain", action="store_true",
                    help="also serve the request stream FIFO on the phased FP64 path (one kernel per phase)")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--profile", action="store_true", help="only run --steps steps of the bench solve (for ncu)")
    ap.add_argument("--profile-n", type=int, default=256, help="grid edge of the --profile solve")
    ap.add_argument("--profile-staging", type=int, default=0,
                    help="PML-shell staging of the --profile solve (0 default ring, 2 TMA tensor copies)")
    ap.add_argument("--profile-batch", action="store_true",
                    help="with --profile: step the 64-scene batch (config 3) instead of the 256^3 solve")
    ap.add_argument("--tile-y", type=int, default=0, help="PML-shell x planes per thread (1, 2, 4; 0 default)")
    ap.add_argument("--x-chunk", type=int, default=0, help="interior x planes per thread (2, 4, 8; 0 default)")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-scene batch (config 3)")
    ap.add_argument("--profile-moving", action="store_true",
                    help="with --profile: step the moving-body solve (config 5) instead of the 256^3 solve")
    ap.add_argument("--no-served", action="store_true", help="skip the serving stream (config 4)")
    ap.add_argument("--no-moving", action="store_true", help="skip the moving-body solve (config 5)")
    ap.add_argument("--serve-rate", type=float, default=4.0)
    ap.add_argument("--serve-requests", type=int, default=16)
    args = ap.parse_args()
    if args.profile:
        return profile_run(args)
    args.warmup = max(3, args.warmup)
    from acoustics_b200 import dist
    ranks = dist.init_from_env()
    world, rank, local = ranks.world, ranks.rank, ranks.local
    if args.impl == "reference":
        rc = run_reference(args, world, rank)
        dist.shutdown(ranks)
        return rc

    import torch

    from acoustics_b200 import scene as S
    from acoustics_b200.solver import PML_WaveSolver

    torch.cuda.set_device(local)
    sc = bench_scene()
    prec = {"fp32": S.PRECISION_FP32_COMPENSATED, "fp64": S.PRECISION_FP64, "fp64-plain": S.PRECISION_FP64}[args.precision]
    kern = S.KERNEL_PHASED if args.precision == "fp64-plain" else S.KERNEL_FUSED
    G = args.graph_steps if args.graph_steps % 2 == 0 else args.graph_steps + 1
    if args.graph_steps == 16 and args.steps % 2 == 0 and 16 < args.steps <= 64:
        # a short timed run replays one graph of its own length (no eager remainder)
        G = args.steps
    K, W = args.steps, args.warmup
    L = sc.n_listeners
    dev_out = torch.empty(max(1, (K + W) * L), dtype=torch.float64, device="cuda")
    solver = PML_WaveSolver(sc, precision=prec, kernel=kern, graph_steps=G, device=local)
    info = solver.info()
    ext = torch.cuda.ExternalStream(solver.stream)
    solver.step_device(W, dev_out.data_ptr())
    solver.prepare_graphs()  # one-time graph capture outside the timed region (runs nothing)
    solver.synchronize()
    dist.barrier(ranks)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        torch.cuda.synchronize()
        e0.record(ext)
        solver.step_device(K, dev_out.data_ptr() + W * L * 8)
        e1.record(ext)
        e1.synchronize()
        torch.cuda.synchronize()
        launches = solver.last_launch_count()
        # kernel-only timing of the dominant step kernel (same stream)
        kernel_ms = solver.time_stencil(K) / K
    ms = e0.elapsed_time(e1)
    dist.barrier(ranks)
    ms_max = dist.max_over_ranks(ms, ranks)
    ms_step = ms_max / K
    value = world * sc.n_cells * K / (ms_max / 1e3) / 1e9
    alg_bytes = float(info.algorithmic_bytes_per_step)
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    kname = {"fp32": "k_ghost_cells<float> || k_interior<float,2> || k_pml_shell_red<float> (reduced PML state)",
             "fp64": "k_ghost_cells<double> || k_interior<double,2> || k_pml_shell<double>",
             "fp64-plain": "phased fp64 (velocity x3, laplacian, pressure)"}[args.precision]
    traffic = read_traffic(args.precision, sc.n_cells)
    clocks = clk.summary()
    y_ours = dev_out[W * L:(W + K) * L].cpu().numpy().reshape(K, L)
    solver.close()

    # end to end through the public API, a whole solve of the configured length
    # (independent of --steps): create (scene tables uploaded, first
    # classification), sc.steps steps with the listener rows copied to host
    # memory, destroy.  Both precisions; their series are the accuracy check.
    def e2e_solve(p2, repeats=2):
        # the whole solve, `repeats` times (host-side costs of a shared machine
        # vary between runs): the fastest is reported, every one is listed
        best, runs, y = None, [], None
        for _ in range(repeats):
            torch.cuda.synchronize()
            dist.barrier(ranks)
            t0 = time.perf_counter()
            s2 = PML_WaveSolver(sc, precision=p2, kernel=S.KERNEL_FUSED, graph_steps=G, device=local)
            t1 = time.perf_counter()
            y = s2.step(sc.steps)
            t2 = time.perf_counter()
            h2d, d2h = s2.transfer_bytes()
            s2.close()
            t3 = time.perf_counter()
            dt = dist.max_over_ranks(t3 - t0, ranks)
            runs.append({"seconds": dt, "create_s": t1 - t0, "steps_s": t2 - t1, "destroy_s": t3 - t2})
            if best is None or dt < best:
                best = dt
        return y, {"value": world * sc.n_cells * sc.steps / best / 1e9, "unit": UNIT,
                   "h2d_bytes_per_step": h2d / sc.steps, "d2h_bytes_per_step": d2h / sc.steps,
                   "steps": sc.steps, "seconds": best, "runs": runs}

    y_e2e32, e2e32 = e2e_solve(S.PRECISION_FP32_COMPENSATED)
    y_e2e64, e2e64 = e2e_solve(S.PRECISION_FP64)
    y_e2e = y_e2e64 if prec == S.PRECISION_FP64 else y_e2e32
    e2e = dict(e2e64 if prec == S.PRECISION_FP64 else e2e32)
    e2e["note"] = (f"whole {sc.steps}-step solve through PML_WaveSolver: create (scene upload, classification), "
                   f"steps with listener rows to host, destroy; the faster of two such solves (runs lists both); "
                   f"bytes counted by fdtd_solver_transfer_bytes")
    # the timed rows must be the rows of the same solve stepped through the public API
    n_cmp = max(0, min(K, sc.steps - W))
    rows_equal = bool(np.array_equal(y_ours[:n_cmp], y_e2e[W:W + n_cmp]))
    fp32_err = float(np.linalg.norm(y_e2e32 - y_e2e64) / np.linalg.norm(y_e2e64))
    checked = {"timed_rows_equal_e2e_rows": rows_equal, "rows_compared": n_cmp,
               "fp32_listener_rel_l2_vs_fp64": fp32_err, "steps": sc.steps,
               "fp32_within_1e-4": fp32_err <= 1e-4,
               "finite": bool(np.all(np.isfinite(y_e2e32)) and np.all(np.isfinite(y_e2e64)))}
    if not (rows_equal and checked["fp32_within_1e-4"] and checked["finite"]):
        print(json.dumps({"error": "bench output check failed", "checked": checked}), flush=True)
        dist.shutdown(ranks)
        return 3

    variants = {"e2e_fp32_compensated": e2e32, "e2e_fp64_fused": e2e64}
    if not args.no_variants:
        for name, p2, k2 in (("fp64_fused", S.PRECISION_FP64, S.KERNEL_FUSED),
                             ("fp64_plain", S.PRECISION_FP64, S.KERNEL_PHASED),
                             ("fp32_compensated", S.PRECISION_FP32_COMPENSATED, S.KERNEL_FUSED)):
            sv = PML_WaveSolver(sc, precision=p2, kernel=k2, graph_steps=G if k2 == S.KERNEL_FUSED else 0, device=local)
            n = min(max(K, 50), 200)
            sv.step_device(5, 0)
            sv.prepare_graphs()
            sv.synchronize()
            ext2 = torch.cuda.ExternalStream(sv.stream)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(ext2)
            sv.step_device(n, 0)
            b.record(ext2)
            b.synchronize()
            t = a.elapsed_time(b) / n
            kms = sv.time_stencil(n) / n
            ab = float(sv.info().algorithmic_bytes_per_step)
            variants[name] = {"gcell_steps_s": sc.n_cells / (t / 1e3) / 1e9, "ms_per_step": t,
                              "kernel_ms": kms, "kernel_hbm_frac": ab / (kms / 1e3) / 1e9 / peak,
                              "alg_bytes_per_step": ab, "steps_timed": n}
            sv.close()
        f32, f64, f64p = (variants[k]["gcell_steps_s"] for k in ("fp32_compensated", "fp64_fused", "fp64_plain"))
        variants["fp32_over_fp64_fused"] = f32 / f64
        variants["fp32_over_fp64_plain"] = f32 / f64p
        variants["note"] = ("fp64_fused is the plain FP64 single-solve path (region-split fused kernels, <=1e-12 "
                            "vs the oracle) and the honest denominator; fp64_plain is one kernel per reference "
                            "phase")

    batched = served = moving = None
    if rank == 0 and world == 1 and not args.no_moving:
        moving = bench_moving(peak)
    if rank == 0 and world == 1 and not args.no_batched:
        batched = bench_batched(peak)
    if rank == 0 and world == 1 and not args.no_served:
        served = bench_served(peak, args.serve_rate, args.serve_requests, fifo_plain=args.fifo_plain)
    if "fp64_fused" in variants:
        # the north-star ratios against the plain FP64 single-solve path
        f64 = variants["fp64_fused"]["gcell_steps_s"]
        if batched:
            batched["over_fp64_fused"] = batched["gcell_steps_s"] / f64
        if served:
            served["over_fp64_fused"] = served["gcell_steps_s"] / f64
            for r in served["rate_sweep"]:
                r["over_fp64_fused"] = r["gcell_steps_s"] / f64

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        val, n, threads, dt = cpu_baseline(sc, args.cpu_budget, 1000)
        cpu = {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{n} full FDTD steps of this 256^3 solve in {dt:.1f} s (FP64 CPU oracle, OpenMP)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp32": "f32", "fp64": "f64", "fp64-plain": "f64"}[args.precision], "data": "synthetic",
            "config": {"workload": sc.name, "cells": sc.n_cells, "divisions": list(sc.divisions),
                       "pml_width": sc.pml_width, "objects": len(sc.objects), "listeners": L,
                       "precision": args.precision, "graph_steps": G,
                       "l2": f"inputs larger than L2: {alg_bytes / 2**20:.0f} MiB algorithmic traffic per step "
                             f"vs {L2_BYTES / 2**20:.0f} MiB L2",
                       "parallelism": f"replicas x{world} (independent solves)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "frac_dram": (traffic / (kernel_ms / 1e3) / 1e9 / peak) if traffic else None,
                         "kernel": kname, "kernel_ms": kernel_ms, "alg_bytes_per_launch": alg_bytes,
                         "note": "frac: algorithmic bytes / CUDA-event time of the step-kernel group; frac_dram: "
                                 "the same with the ncu DRAM bytes of that group (traffic)"},
            "e2e": e2e,
            "checked": checked,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "variants": variants,
        }
        if batched:
            line["batched"] = batched
        if served:
            line["served"] = served
        if moving:
            line["moving"] = moving
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    dist.shutdown(ranks)
    return 0


if __name__ == "__main__":
    sys.exit(main())
