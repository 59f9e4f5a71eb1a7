"""ctypes binding of the FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  The oracle is the checker; the product library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from acoustics_b200.scene import CELL_DTYPE, GHOST_FACE_DTYPE, GhostFace, Scene

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.oracle_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.oracle_create.restype = C.c_int
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_reset.argtypes = [C.c_void_p, C.c_double]
        L.oracle_step.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.oracle_step.restype = C.c_int
        L.oracle_time.argtypes = [C.c_void_p]
        L.oracle_time.restype = C.c_double
        L.oracle_num_cells.argtypes = [C.c_void_p]
        L.oracle_num_cells.restype = C.c_int64
        L.oracle_num_pml_cells.argtypes = [C.c_void_p]
        L.oracle_num_pml_cells.restype = C.c_int64
        L.oracle_get_classification.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]
        L.oracle_get_classification.restype = C.c_int
        L.oracle_get_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64]
        L.oracle_get_field.restype = C.c_int
        L.oracle_fetch_listeners.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_fetch_listeners.restype = C.c_int
        L.oracle_fetch_cell.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        L.oracle_fetch_cell.restype = C.c_int
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_set_threads.restype = C.c_int
        L.oracle_mls_c0.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        L.oracle_mls_c0.restype = C.c_int
        L.oracle_mesh_sdf.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p]
        L.oracle_mesh_sdf.restype = C.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return lib().oracle_set_threads(int(n))


class OracleSolver:
    """FP64 CPU restatement of PML_WaveSolver + the SimWorld listener loop."""

    def __init__(self, scene: Scene):
        self.scene = scene
        desc, self._keep = scene.to_c()
        h = C.c_void_p()
        st = lib().oracle_create(C.byref(desc), C.byref(h))
        if st != 0:
            raise RuntimeError(f"oracle_create failed with status {st}")
        self._h = h
        self.L = scene.n_listeners
        self.n_cells = int(lib().oracle_num_cells(h))

    def close(self):
        if getattr(self, "_h", None):
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def reset(self, t0: float = 0.0):
        lib().oracle_reset(self._h, t0)

    def step(self, n: int) -> np.ndarray:
        out = np.zeros((n, max(self.L, 1)), dtype=np.float64)
        st = lib().oracle_step(self._h, int(n), out.ctypes.data)
        if st not in (0, 1, -4):
            raise RuntimeError(f"oracle_step failed with status {st}")
        self.last_status = st
        return out[:, : self.L]

    @property
    def time(self) -> float:
        return lib().oracle_time(self._h)

    @property
    def n_pml_cells(self) -> int:
        return int(lib().oracle_num_pml_cells(self._h))

    def classification(self):
        flags = np.zeros(self.n_cells, dtype=np.uint8)
        n = C.c_int64(0)
        lib().oracle_get_classification(self._h, flags.ctypes.data, None, C.byref(n))
        faces = np.zeros(n.value, dtype=GHOST_FACE_DTYPE)
        cap = C.c_int64(n.value)
        lib().oracle_get_classification(self._h, None, faces.ctypes.data, C.byref(cap))
        return flags, faces

    def field(self, which: int) -> np.ndarray:
        N = [int(x) for x in self.scene.divisions]
        if which <= 4:
            count = N[0] * N[1] * N[2]
        else:
            d = which - 5
            N[d] += 1
            count = N[0] * N[1] * N[2]
        out = np.zeros(count, dtype=np.float64)
        st = lib().oracle_get_field(self._h, int(which), out.ctypes.data, count)
        if st != 0:
            raise RuntimeError(f"oracle_get_field failed {st}")
        return out

    def fetch_cell(self, cell_index: int) -> np.void:
        """MAC_Grid::GetCell + the stored Laplacian, a record of CELL_DTYPE."""
        out = np.zeros(1, dtype=CELL_DTYPE)
        st = lib().oracle_fetch_cell(self._h, int(cell_index), out.ctypes.data)
        if st != 0:
            raise RuntimeError(f"oracle_fetch_cell failed {st}")
        return out[0]

    def fetch_listeners(self) -> np.ndarray:
        out = np.zeros(max(self.L, 1))
        lib().oracle_fetch_listeners(self._h, out.ctypes.data)
        return out[: self.L]


def mls_c0(p, pts, vals) -> float:
    p = np.ascontiguousarray(p, dtype=np.float64)
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    out = C.c_double(0.0)
    st = lib().oracle_mls_c0(p.ctypes.data, pts.ctypes.data, vals.ctypes.data, len(vals), C.byref(out))
    if st != 0:
        raise RuntimeError("rank-deficient MLS stencil")
    return out.value
