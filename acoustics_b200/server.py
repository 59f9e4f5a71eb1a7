"""Solve server: continuous batching of submitted scenes on one GPU.

The reference steps one scene per process (src/wavesolver/SimWorld.cpp:517-590);
`SolveServer` accepts scenes at any time, admits them in arrival order while
their device bytes fit the budget, keeps their grids resident and steps all
admitted scenes together (fdtd_server_* in include/fdtd_c.h).  A request's
listener series equals that of `PML_WaveSolver` on the same scene and options.
Requests can be cancelled; with `preempt` a queue head that does not fit evicts
members with much more work left to host memory (the reference's snapshot,
FDTD_AcousticSimulator.cpp:381-415), which resume where they stopped.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Tuple

import numpy as np

from ._lib import FDTDError, check, load
from .scene import (KERNEL_FUSED, PRECISION_FP32_COMPENSATED, REQ_CANCELLED, REQ_DONE, REQ_FAILED, Options, Scene,
                    ServerConfig, ServerStats)


class SolveServer:
    def __init__(self, precision: int = PRECISION_FP32_COMPENSATED, graph_steps: int = 16, device: int = 0,
                 hbm_budget_bytes: int = 0, max_members: int = 0, chunk_steps: int = 0, tile_y: int = 0,
                 x_chunk: int = 0, preempt: bool = False, tune_for=None):
        """`tune_for`: scenes typical of the requests; with `tile_y` / `x_chunk` 0 the
        batched step uses the autotuned shapes of their grid class."""
        self._L = load()
        if tune_for and tile_y == 0 and x_chunk == 0:
            from .autotune import shapes_for
            x_chunk, tile_y = shapes_for(list(tune_for), precision, device=device)
        self.shape = (x_chunk, tile_y)
        opt = Options(precision=precision, device=device, kernel=KERNEL_FUSED, graph_steps=graph_steps,
                      tile_y=tile_y, x_chunk=x_chunk)
        cfg = ServerConfig(hbm_budget_bytes=int(hbm_budget_bytes), max_members=int(max_members),
                           chunk_steps=int(chunk_steps), preempt=1 if preempt else 0)
        h = C.c_void_p()
        check(self._L.fdtd_server_create(C.byref(opt), C.byref(cfg), C.byref(h)))
        self._h = h

    def submit(self, scene: Scene, steps: int = 0) -> int:
        desc, keep = scene.to_c()
        rid = C.c_int64(0)
        check(self._L.fdtd_server_submit(self._h, C.byref(desc), int(steps or scene.steps), C.byref(rid)))
        del keep
        return int(rid.value)

    def poll(self, rid: int) -> Tuple[int, int, int]:
        """(state REQ_*, steps done, status)"""
        st, done, status = C.c_int32(), C.c_int64(), C.c_int32()
        check(self._L.fdtd_server_poll(self._h, int(rid), C.byref(st), C.byref(done), C.byref(status)))
        return int(st.value), int(done.value), int(status.value)

    def wait(self, rid: int, timeout_s: float = -1.0):
        st = self._L.fdtd_server_wait(self._h, int(rid), float(timeout_s))
        if st < 0:
            msg = (self._L.fdtd_server_request_error(self._h, int(rid)) or b"").decode() or \
                  (self._L.fdtd_last_error() or b"").decode()
            raise FDTDError(st, msg)

    def result(self, rid: int) -> Tuple[np.ndarray, float]:
        """(series of shape (steps, n_listeners), latency in s); the request is forgotten."""
        self.wait(rid)
        steps, nl, lat = C.c_int64(), C.c_int32(), C.c_double()
        check(self._L.fdtd_server_result(self._h, int(rid), None, 0, C.byref(steps), C.byref(nl), C.byref(lat)))
        buf = np.zeros(max(1, steps.value * nl.value), dtype=np.float64)
        check(self._L.fdtd_server_result(self._h, int(rid), buf.ctypes.data, buf.size, None, None, C.byref(lat)))
        return buf[: steps.value * nl.value].reshape(steps.value, nl.value), float(lat.value)

    def cancel(self, rid: int):
        """Cancel a queued or running request (its wait / result raise FDTD_ERR_CANCELLED)."""
        check(self._L.fdtd_server_cancel(self._h, int(rid)))

    def drain(self, timeout_s: float = -1.0):
        check(self._L.fdtd_server_drain(self._h, float(timeout_s)))

    def stats(self) -> Dict[str, float]:
        s = ServerStats()
        check(self._L.fdtd_server_stats_get(self._h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            self._L.fdtd_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


__all__ = ["SolveServer", "REQ_DONE", "REQ_FAILED", "REQ_CANCELLED"]
