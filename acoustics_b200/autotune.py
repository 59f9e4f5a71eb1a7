"""Autotuner of the batched step's tile shapes, cached per grid class.

The batched step (fdtd_batch_*) has two shape knobs that do not change any
result bit (every FP32 kernel requests its FMAs explicitly and the units are
built without contraction): the x planes an interior thread updates
(`x_chunk`: 2, 4, 8) and the x planes a PML-shell thread marches over
(`tile_y`: 4, 8, 16).  Which is fastest depends on the grids: small boxes
leave partial tiles, PML-heavy grids spend their time in the shell.  The
tuner times every candidate on a sample of the scenes of a grid class (CUDA
events on the batch stream, after warm-up steps) and caches the fastest per
class in a JSON file; `SolveBatch` and `SolveServer` look their class up
there (and tune on a miss) unless shapes are given explicitly.

A grid class is (precision, GPU name, bucket of log2 of the mean cell count,
bucket of the mean PML fraction).  The cache lives in $FDTD_TUNE_CACHE, else in
~/.cache/acoustics_b200/tuned_shapes.json.  The reference runs fixed OpenMP
loops and has nothing to tune (src/wavesolver/MAC_Grid.cpp:197, :465).
"""
from __future__ import annotations

import copy
import json
import math
import os
import threading
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .scene import PRECISION_FP32_COMPENSATED, PRECISION_FP64, Scene

X_CHUNKS = (2, 4, 8)
TILE_YS = (4, 8, 16)
DEFAULT_SHAPE = (2, 8)
_lock = threading.Lock()


def cache_path() -> str:
    p = os.environ.get("FDTD_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "acoustics_b200", "tuned_shapes.json")


def pml_fraction(sc: Scene) -> float:
    return sc.n_pml_cells() / max(1, sc.n_cells)


def grid_class(scenes: Sequence[Scene], precision: int, device_name: str = "") -> str:
    """Key of the grid class of a set of scenes."""
    cells = float(np.mean([sc.n_cells for sc in scenes])) if scenes else 1.0
    frac = float(np.mean([pml_fraction(sc) for sc in scenes])) if scenes else 0.0
    prec = "fp64" if precision == PRECISION_FP64 else "fp32"
    return f"{prec}|{device_name or 'gpu'}|cells2^{int(round(math.log2(max(cells, 1.0))))}|pml{int(frac * 10)}"


def load_cache(path: Optional[str] = None) -> Dict[str, dict]:
    path = path or cache_path()
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def store(key: str, entry: dict, path: Optional[str] = None) -> None:
    path = path or cache_path()
    with _lock:
        d = load_cache(path)
        d[key] = entry
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        tmp = path + f".tmp{os.getpid()}"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def lookup(scenes: Sequence[Scene], precision: int, device_name: str = "",
           path: Optional[str] = None) -> Optional[Tuple[int, int]]:
    e = load_cache(path).get(grid_class(scenes, precision, device_name))
    if not e:
        return None
    return int(e["x_chunk"]), int(e["tile_y"])


def device_name(device: int = 0) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device).replace(" ", "_")
    except Exception:
        return "gpu"


def _sample(scenes: Sequence[Scene], n: int, steps: int) -> List[Scene]:
    """Up to n scenes spread over the set (sorted by size), each long enough to
    stay active through the timed steps."""
    order = sorted(range(len(scenes)), key=lambda i: scenes[i].n_cells)
    pick = [order[int(round(k * (len(order) - 1) / max(1, n - 1)))] for k in range(min(n, len(order)))]
    out = []
    for i in sorted(set(pick)):
        sc = copy.deepcopy(scenes[i])
        sc.steps = steps
        out.append(sc)
    return out


def time_shape(scenes: Sequence[Scene], precision: int, x_chunk: int, tile_y: int, steps: int = 48,
               warmup: int = 16, graph_steps: int = 16, device: int = 0) -> float:
    """Milliseconds per batched step of `scenes` with one shape (CUDA events on the batch stream)."""
    import torch

    from .batch import SolveBatch
    with SolveBatch(scenes, precision=precision, graph_steps=graph_steps, device=device, x_chunk=x_chunk,
                    tile_y=tile_y, tune=False) as b:
        b.step(warmup)
        ext = torch.cuda.ExternalStream(b.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(ext)
        b.step(steps)
        e1.record(ext)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps


def tune(scenes: Sequence[Scene], precision: int = PRECISION_FP32_COMPENSATED, sample: int = 12,
         steps: int = 48, graph_steps: int = 16, device: int = 0, path: Optional[str] = None,
         candidates: Optional[Sequence[Tuple[int, int]]] = None) -> dict:
    """Time every candidate shape on a sample of `scenes`, cache and return the
    entry {x_chunk, tile_y, ms_per_step, timings, ...} of their grid class."""
    cand = list(candidates) if candidates else [(x, t) for x in X_CHUNKS for t in TILE_YS]
    smp = _sample(scenes, sample, steps + 64)
    timings = {}
    for x, t in cand:
        timings[f"{x}x{t}"] = time_shape(smp, precision, x, t, steps=steps, graph_steps=graph_steps, device=device)
    best = min(timings, key=timings.get)
    x, t = (int(v) for v in best.split("x"))
    name = device_name(device)
    key = grid_class(scenes, precision, name)
    entry = {"x_chunk": x, "tile_y": t, "ms_per_step": timings[best], "timings_ms": timings,
             "sample_scenes": len(smp), "sample_cells": int(sum(sc.n_cells for sc in smp)),
             "default_ms_per_step": timings.get(f"{DEFAULT_SHAPE[0]}x{DEFAULT_SHAPE[1]}")}
    store(key, entry, path)
    entry["key"] = key
    return entry


def shapes_for(scenes: Sequence[Scene], precision: int, device: int = 0, tune_on_miss: bool = True,
               path: Optional[str] = None) -> Tuple[int, int]:
    """Cached shape of the grid class of `scenes`; on a miss, tune it now (when
    allowed) or return the defaults."""
    if not scenes:
        return DEFAULT_SHAPE
    name = device_name(device)
    hit = lookup(scenes, precision, name, path)
    if hit:
        return hit
    if not tune_on_miss:
        return DEFAULT_SHAPE
    e = tune(scenes, precision, device=device, path=path)
    return e["x_chunk"], e["tile_y"]
