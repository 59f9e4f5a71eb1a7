"""Multi-GPU serving: one solve server per GPU, requests routed between them.

The path shards across solves, not within one, so the GPUs share no data: a
router keeps one `SolveServer` per device and sends each request to the device
with the least outstanding work (cells x steps of its routed, unfinished
requests) among those whose device-byte budget can hold the request's
footprint.  No collective and no inter-GPU traffic; each server admits,
batches and retires its own requests.  The reference runs one solve per
process (src/wavesolver/SimWorld.cpp:517-590) and has no server.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from .scene import PRECISION_FP32_COMPENSATED, Scene


class ServerRouter:
    def __init__(self, devices: Optional[Sequence[int]] = None, precision: int = PRECISION_FP32_COMPENSATED,
                 hbm_budget_bytes: int = 0, server_factory: Optional[Callable] = None,
                 footprint: Optional[Callable[[Scene], int]] = None, **server_kw):
        """`server_factory(device=d, precision=..., hbm_budget_bytes=..., **server_kw)`
        makes the per-device server (default: SolveServer); `footprint(scene)` is
        a request's device bytes (default: the library's estimate)."""
        if devices is None:
            from .solver import device_count
            devices = list(range(device_count()))
        if not devices:
            raise ValueError("no device to serve on")
        if server_factory is None:
            from .server import SolveServer
            server_factory = SolveServer
        if footprint is None:
            from .batch import scene_device_bytes

            def footprint(sc):
                return scene_device_bytes(sc, precision=precision)
        self.devices = list(devices)
        self.footprint = footprint
        self.servers = [server_factory(device=d, precision=precision, hbm_budget_bytes=hbm_budget_bytes, **server_kw)
                        for d in self.devices]
        self.budget = [int(hbm_budget_bytes) if hbm_budget_bytes > 0 else None for _ in self.devices]
        self.work = [0.0] * len(self.devices)     # outstanding cells x steps per device
        self.routed: Dict[Tuple[int, int], float] = {}
        self.counts = [0] * len(self.devices)

    def route(self, scene: Scene, steps: int) -> int:
        """Index of the server a request goes to."""
        need = self.footprint(scene)
        fits = [i for i in range(len(self.servers)) if self.budget[i] is None or need <= self.budget[i]]
        if not fits:
            raise ValueError(f"the request needs {need} device bytes, more than any device's budget")
        return min(fits, key=lambda i: (self.work[i], i))

    def submit(self, scene: Scene, steps: int = 0) -> Tuple[int, int]:
        steps = int(steps or scene.steps)
        i = self.route(scene, steps)
        rid = self.servers[i].submit(scene, steps)
        w = float(scene.n_cells) * steps
        self.work[i] += w
        self.routed[(i, rid)] = w
        self.counts[i] += 1
        return (i, rid)

    def _done(self, key: Tuple[int, int]):
        w = self.routed.pop(key, 0.0)
        self.work[key[0]] -= w

    def result(self, key: Tuple[int, int]):
        """(series, latency) of a request; its work leaves the device's account."""
        try:
            return self.servers[key[0]].result(key[1])
        finally:
            self._done(key)

    def cancel(self, key: Tuple[int, int]):
        self.servers[key[0]].cancel(key[1])
        self._done(key)

    def stats(self) -> List[dict]:
        out = []
        for i, s in enumerate(self.servers):
            st = dict(s.stats())
            st["device"] = self.devices[i]
            st["routed"] = self.counts[i]
            st["outstanding_cell_steps"] = self.work[i]
            out.append(st)
        return out

    def close(self):
        for s in self.servers:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def balance(work: Sequence[float]) -> float:
    """max / mean of per-device work (1.0: perfectly even)."""
    w = np.asarray(work, dtype=np.float64)
    return float(w.max() / w.mean()) if w.size and w.mean() > 0 else 1.0
