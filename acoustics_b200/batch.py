"""Many independent static solves stepped together on one GPU.

The reference runs its sim units one after another (src/wavesolver/SimWorld.cpp:517-590);
`SolveBatch` keeps every member resident and advances all of them per step
with a fixed number of kernel launches (fdtd_batch_* in include/fdtd_c.h).
Each member's listener series equals the one `PML_WaveSolver` produces for the
same scene and options.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from ._lib import check, load
from .scene import KERNEL_FUSED, PRECISION_FP32_COMPENSATED, Options, Scene


def scene_device_bytes(scene: Scene, precision: int = PRECISION_FP32_COMPENSATED, kernel: int = KERNEL_FUSED,
                       graph_steps: int = 0) -> int:
    """Device bytes a solver of `scene` allocates (admission by HBM footprint)."""
    L = load()
    desc, keep = scene.to_c()
    opt = Options(precision=precision, kernel=kernel, graph_steps=graph_steps)
    n = int(L.fdtd_scene_device_bytes(C.byref(desc), C.byref(opt)))
    del keep
    if n < 0:
        check(-1)
    return n


def scene_info(scene: Scene, precision: int = PRECISION_FP32_COMPENSATED, kernel: int = KERNEL_FUSED):
    """SolverInfo of a solver of `scene` (cell counts, device and algorithmic bytes), host only."""
    from .scene import SolverInfo
    L = load()
    desc, keep = scene.to_c()
    opt = Options(precision=precision, kernel=kernel)
    info = SolverInfo()
    check(L.fdtd_scene_info(C.byref(desc), C.byref(opt), C.byref(info)))
    del keep
    return info


class SolveBatch:
    def __init__(self, scenes: Sequence[Scene] = (), steps: Optional[Sequence[int]] = None,
                 precision: int = PRECISION_FP32_COMPENSATED, graph_steps: int = 16, device: int = 0,
                 tile_y: int = 0, x_chunk: int = 0, tune: bool = True):
        """`tile_y` / `x_chunk` 0 with `tune`: the autotuned shapes of the grid
        class of `scenes` (acoustics_b200.autotune; tuned now on a cache miss)."""
        self._L = load()
        if tune and scenes and tile_y == 0 and x_chunk == 0:
            from .autotune import shapes_for
            x_chunk, tile_y = shapes_for(list(scenes), precision, device=device)
        self.shape = (x_chunk, tile_y)
        opt = Options(precision=precision, device=device, kernel=KERNEL_FUSED, graph_steps=graph_steps,
                      tile_y=tile_y, x_chunk=x_chunk)
        h = C.c_void_p()
        check(self._L.fdtd_batch_create(0, None, None, C.byref(opt), C.byref(h)))
        self._h = h
        self.scenes: List[Scene] = []
        for i, sc in enumerate(scenes):
            self.add(sc, int(steps[i] if steps is not None else sc.steps))

    def add(self, scene: Scene, steps: int) -> int:
        """Add a member; its first (classifying) step runs at once.  Returns its index."""
        desc, keep = scene.to_c()
        m = C.c_int32(-1)
        check(self._L.fdtd_batch_add(self._h, C.byref(desc), int(steps), C.byref(m)))
        del keep
        self.scenes.append(scene)
        return int(m.value)

    def step(self, n: int) -> int:
        """Advance every active member by up to n steps; returns the members still running."""
        a = C.c_int32(0)
        check(self._L.fdtd_batch_step(self._h, int(n), C.byref(a)))
        return int(a.value)

    def run(self):
        check(self._L.fdtd_batch_run(self._h))

    def info(self, m: int):
        done, total, nl, st = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
        check(self._L.fdtd_batch_member_info(self._h, int(m), C.byref(done), C.byref(total), C.byref(nl),
                                             C.byref(st)))
        return int(done.value), int(total.value), int(nl.value), int(st.value)

    def output(self, m: int) -> np.ndarray:
        """Listener series of member m so far, shape (steps_done, n_listeners)."""
        done, _, nl, st = self.info(m)
        out = np.zeros((done, nl), dtype=np.float64)
        check(self._L.fdtd_batch_output(self._h, int(m), out.ctypes.data if out.size else None, out.size))
        check(st)
        return out

    def release(self, m: int):
        check(self._L.fdtd_batch_release(self._h, int(m)))

    @property
    def stream(self) -> int:
        return int(self._L.fdtd_batch_stream(self._h) or 0)

    def last_launch_count(self) -> int:
        return int(self._L.fdtd_batch_last_launch_count(self._h))

    def device_bytes(self) -> int:
        return int(self._L.fdtd_batch_device_bytes(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self._L.fdtd_batch_destroy(self._h)
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
