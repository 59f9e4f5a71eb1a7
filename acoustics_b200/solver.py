"""Host-side mirror of the reference's solver interface.

`PML_WaveSolver` keeps the member names of src/wavesolver/PML_WaveSolver.h
(stepSystem, FetchPressureData, Reinitialize_PML_WaveSolver, GetGrid) and
`FDTD_AcousticSimulator` those of src/wavesolver/FDTD_AcousticSimulator.h
(InitializeSolver, RunForSteps, Run, GetSolver).  Both drive the CUDA library
through the C-ABI of include/fdtd_c.h; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from ._lib import FDTDError, check, load
from .scene import (CELL_DTYPE, FIELD_PRESSURE, GHOST_FACE_DTYPE, KERNEL_FUSED, PML_STATE_AUTO, PRECISION_FP64, Options,
                    Scene, SceneDesc, SolverInfo)


class PML_WaveSolver:
    """One resident solve on one GPU (PML_WaveSolver.h:122-255)."""

    def __init__(self, scene: Scene, precision: int = PRECISION_FP64, kernel: int = KERNEL_FUSED,
                 graph_steps: int = 0, device: int = 0, tile_y: int = 0, x_chunk: int = 0,
                 pml_state: int = PML_STATE_AUTO, shell_staging: int = 0):
        self._L = load()
        self.scene = scene
        desc, self._keep = scene.to_c()
        opt = Options(precision=precision, device=device, kernel=kernel, graph_steps=graph_steps,
                      tile_y=tile_y, x_chunk=x_chunk, pml_state=pml_state, shell_staging=shell_staging)
        h = C.c_void_p()
        check(self._L.fdtd_solver_create(C.byref(desc), C.byref(opt), C.byref(h)))
        self._h = h
        self.precision = precision
        self.n_listeners = scene.n_listeners
        info = self.info()
        self.divisions = tuple(info.divisions)
        self.n_cells = int(info.n_cells)

    # ---- lifecycle ----
    def close(self):
        if getattr(self, "_h", None):
            self._L.fdtd_solver_destroy(self._h)
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

    def pml_state(self) -> int:
        """PML_STATE_AUTO when this solve keeps the reduced PML state, else PML_STATE_FULL."""
        return int(self._L.fdtd_solver_pml_state(self._h))

    def shell_staging(self) -> int:
        """SHELL_STAGING_TMA or SHELL_STAGING_RING for the reduced-state PML shell in
        effect, -1 when the solve keeps the full PML state."""
        return int(self._L.fdtd_solver_shell_staging(self._h))

    def Reinitialize_PML_WaveSolver(self, start_time: float = 0.0):
        check(self._L.fdtd_solver_reset(self._h, float(start_time)), self._h)

    # ---- stepping ----
    def step(self, n: int, record: bool = True) -> np.ndarray:
        """n x (stepSystem + FetchPressureData): listener series, shape (n, L)."""
        out = np.zeros((n, max(1, self.n_listeners)), dtype=np.float64) if record else None
        st = self._L.fdtd_solver_step(self._h, int(n), out.ctypes.data if record else None)
        check(st, self._h)
        self.last_status = st
        return out[:, : self.n_listeners] if record else None

    def step_device(self, n: int, device_ptr: int) -> int:
        return check(self._L.fdtd_solver_step_device(self._h, int(n), C.c_void_p(device_ptr)), self._h)

    def stepSystem(self) -> bool:
        """One step; False once the end time is reached (PML_WaveSolver.cpp:579-609)."""
        st = self._L.fdtd_solver_step(self._h, 1, None)
        check(st, self._h)
        return st != 1

    def FetchPressureData(self) -> np.ndarray:
        """Listener values at the current state (PML_WaveSolver.cpp:319-373)."""
        out = np.zeros(max(1, self.n_listeners))
        check(self._L.fdtd_solver_fetch_listeners(self._h, out.ctypes.data), self._h)
        return out[: self.n_listeners]

    def synchronize(self):
        check(self._L.fdtd_solver_synchronize(self._h), self._h)

    @property
    def stream(self) -> int:
        return int(self._L.fdtd_solver_stream(self._h) or 0)

    def last_launch_count(self) -> int:
        return int(self._L.fdtd_solver_last_launch_count(self._h))

    def overlapped_steps(self) -> int:
        """Steps whose PML-shell kernel ran beside the step's cell classification
        (moving bodies clear of the PML); execution statistics only."""
        return int(self._L.fdtd_solver_overlapped_steps(self._h))

    def transfer_bytes(self):
        """(host-to-device, device-to-host) bytes this solve has copied since creation."""
        a, b = C.c_int64(0), C.c_int64(0)
        check(self._L.fdtd_solver_transfer_bytes(self._h, C.byref(a), C.byref(b)), self._h)
        return int(a.value), int(b.value)

    def prepare_graphs(self):
        """Capture the CUDA graph of the next graph_steps-long chunk now (nothing runs)."""
        check(self._L.fdtd_solver_prepare_graphs(self._h), self._h)

    def time_stencil(self, n_launches: int) -> float:
        """Milliseconds for n back-to-back launches of the step kernel (CUDA events
        on the solver stream).  Advances the state without prologue/listeners."""
        ms = C.c_float(0.0)
        check(self._L.fdtd_solver_time_stencil(self._h, int(n_launches), C.byref(ms)), self._h)
        return float(ms.value)

    def time_kernel(self, which: int, n_launches: int) -> float:
        """Milliseconds for n launches of one part of the step: 0 step kernels,
        1 interior, 2 PML shell, 3 ghost-cell list, 4 listeners (timing only)."""
        ms = C.c_float(0.0)
        check(self._L.fdtd_solver_time_kernel(self._h, int(which), int(n_launches), C.byref(ms)), self._h)
        return float(ms.value)

    # ---- introspection ----
    def info(self) -> SolverInfo:
        info = SolverInfo()
        check(self._L.fdtd_solver_info_get(self._h, C.byref(info)), self._h)
        return info

    @property
    def time(self) -> float:
        return float(self.info().time)

    def GetGrid(self):
        """(flags[N] uint8, ghost faces) after the last classification (MAC_Grid.h:372-484)."""
        flags = np.zeros(self.n_cells, dtype=np.uint8)
        n = C.c_int64(0)
        check(self._L.fdtd_solver_get_classification(self._h, flags.ctypes.data, None, C.byref(n)), self._h)
        faces = np.zeros(n.value, dtype=GHOST_FACE_DTYPE)
        cap = C.c_int64(n.value)
        check(self._L.fdtd_solver_get_classification(self._h, None, faces.ctypes.data, C.byref(cap)), self._h)
        return flags, faces

    def GetSolverDomain(self):
        """(min_bound, max_bound) of the pressure grid (PML_WaveSolver.cpp:458-471)."""
        lo, hi = np.zeros(3), np.zeros(3)
        check(self._L.fdtd_solver_domain(self._h, lo.ctypes.data, hi.ctypes.data), self._h)
        return lo, hi

    def FetchCell(self, cell_index: int) -> np.void:
        """One cell as MAC_Grid::GetCell fills it, plus the stored Laplacian
        (PML_WaveSolver.cpp:439-447); a record of CELL_DTYPE."""
        out = np.zeros(1, dtype=CELL_DTYPE)
        check(self._L.fdtd_solver_fetch_cell(self._h, int(cell_index), out.ctypes.data), self._h)
        return out[0]

    def SampleAxisAlignedSlice(self, dim: int, offset: float) -> np.ndarray:
        """The cells of the plane across axis `dim` at `offset` (MAC_Grid.cpp:1941-1963),
        an array of CELL_DTYPE in the reference's order."""
        n = C.c_int64(0)
        check(self._L.fdtd_solver_sample_slice(self._h, int(dim), float(offset), None, 0, C.byref(n)), self._h)
        out = np.zeros(n.value, dtype=CELL_DTYPE)
        check(self._L.fdtd_solver_sample_slice(self._h, int(dim), float(offset), out.ctypes.data, out.size,
                                               C.byref(n)), self._h)
        return out

    def field(self, which: int = FIELD_PRESSURE) -> np.ndarray:
        N = list(self.divisions)
        if which >= 5:
            N[which - 5] += 1
        count = N[0] * N[1] * N[2]
        out = np.zeros(count, dtype=np.float64)
        check(self._L.fdtd_solver_get_field(self._h, int(which), out.ctypes.data, count), self._h)
        return out

    def boundary_info(self) -> dict:
        """FULLY_COUPLED rows (total, immersed, fallen back) and the last solve's iterations."""
        a, b, c, d = C.c_int64(0), C.c_int64(0), C.c_int64(0), C.c_int32(0)
        check(self._L.fdtd_solver_boundary_info(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)), self._h)
        return {"rows": a.value, "immersed": b.value, "fallback": c.value, "iterations": d.value}

    def set_field(self, which: int, values) -> None:
        """The inverse of field(): a dense field (the reference's flat order) into the solve."""
        a = np.ascontiguousarray(values, dtype=np.float64).ravel()
        check(self._L.fdtd_solver_set_field(self._h, int(which), a.ctypes.data, a.size), self._h)

    # ---- the reference's output files (FDTD_AcousticSimulator.cpp) ----
    def save_snapshot(self, numbering: str, output_pattern: str = "%s") -> None:
        """_SaveSimulationSnapshot(numbering): snapshot_<numbering>_*.dat files."""
        check(self._L.fdtd_solver_save_snapshot(self._h, output_pattern.encode(), str(numbering).encode()), self._h)

    def load_snapshot(self, numbering: str, output_pattern: str = "%s") -> None:
        check(self._L.fdtd_solver_load_snapshot(self._h, output_pattern.encode(), str(numbering).encode()), self._h)

    def save_config(self, output_pattern: str = "%s") -> None:
        """SaveSolverConfig's position files."""
        check(self._L.fdtd_solver_save_config(self._h, output_pattern.encode()), self._h)

    def save_field_timestep(self, path: str, which: int = FIELD_PRESSURE) -> None:
        """_SavePressureTimestep / _SaveVelocityTimestep: (n x 1) matrix, x fastest."""
        check(self._L.fdtd_solver_save_field_timestep(self._h, int(which), path.encode()), self._h)

    def snapshot(self) -> bytes:
        n = C.c_int64(0)
        check(self._L.fdtd_solver_snapshot(self._h, None, C.byref(n)), self._h)
        buf = (C.c_char * n.value)()
        check(self._L.fdtd_solver_snapshot(self._h, buf, C.byref(n)), self._h)
        return bytes(buf)

    def restore(self, blob: bytes):
        buf = C.create_string_buffer(blob, len(blob))
        check(self._L.fdtd_solver_restore(self._h, buf, len(blob)), self._h)


def scene_from_xml(path: str) -> Scene:
    """Read an <impulse_response> XML scene through the library's reader."""
    L = load()
    h = C.c_void_p()
    check(L.fdtd_scene_from_xml(path.encode(), C.byref(h)))
    try:
        d = L.fdtd_scene_desc_get(h).contents
        from .scene import GaussianSource, PlaneConstraint, RigidObject, TriangleMesh
        sc = Scene(cell_size=d.cell_size, divisions=tuple(d.divisions), time_step=d.time_step,
                   domain_center=tuple(d.domain_center), sound_speed=d.sound_speed, density=d.density,
                   pml_width=d.pml_width, pml_strength=d.pml_strength,
                   boundary_condition_preset=d.boundary_condition_preset,
                   air_viscosity_alpha=d.air_viscosity_alpha, start_time=d.start_time, end_time=d.end_time,
                   boundary_handling=d.boundary_handling)
        for i in range(d.n_objects):
            o = d.objects[i]
            sc.objects.append(RigidObject(o.shape, tuple(o.center), tuple(o.size), tuple(o.rotation), o.accel_kind,
                                          o.accel_amplitude, o.accel_t0, o.accel_tau, tuple(o.accel_dir), o.motion,
                                          tuple(o.velocity), tuple(o.gravity), int(o.mesh)))
        for i in range(d.n_meshes):
            m = d.meshes[i]
            v = np.ctypeslib.as_array(m.vertices, shape=(m.n_vertices * 3,)).reshape(-1, 3).copy()
            t = np.ctypeslib.as_array(m.triangles, shape=(m.n_triangles * 3,)).reshape(-1, 3).copy()
            sc.meshes.append(TriangleMesh(v, t))
        from .scene import KeyframeTrack
        for i in range(d.n_tracks):
            t = d.tracks[i]
            fr = np.ctypeslib.as_array(t.frames, shape=(t.n_frames * 7,)).reshape(-1, 7).copy()
            sc.tracks.append(KeyframeTrack(int(t.object), float(t.step), fr))
        for i in range(d.n_constraints):
            p = d.constraints[i]
            sc.constraints.append(PlaneConstraint(p.normal_dir, p.normal_sign, p.height))
        for i in range(d.n_sources):
            s = d.sources[i]
            sc.sources.append(GaussianSource(tuple(s.position), s.width_time, s.width_space, s.offset_time,
                                             s.normalize_constant))
        if d.n_listeners:
            sc.listeners = np.ctypeslib.as_array(d.listeners, shape=(d.n_listeners * 3,)).reshape(-1, 3).copy()
        sc.steps = int(L.fdtd_scene_number_of_steps(h))
        sc.output_pattern = (L.fdtd_scene_output_pattern(h) or b"%s").decode()
        return sc
    finally:
        L.fdtd_scene_free(h)


class FDTD_AcousticSimulator:
    """Façade of FDTD_AcousticSimulator (FDTD_AcousticSimulator.cpp:419-621) with the
    headless TUI_Run loop and the all_audio.dat listener output of SimWorld/AudioOutput."""

    def __init__(self, scene_or_xml, precision: int = PRECISION_FP64, graph_steps: int = 0, device: int = 0):
        self.scene = scene_from_xml(scene_or_xml) if isinstance(scene_or_xml, str) else scene_or_xml
        self.precision = precision
        self.graph_steps = graph_steps
        self.device = device
        self._solver: Optional[PML_WaveSolver] = None

    def InitializeSolver(self):
        self._solver = PML_WaveSolver(self.scene, precision=self.precision, graph_steps=self.graph_steps,
                                      device=self.device)
        return self._solver

    def GetSolver(self) -> PML_WaveSolver:
        if self._solver is None:
            self.InitializeSolver()
        return self._solver

    def ResetStartTime(self, start_time: float):
        self.GetSolver().Reinitialize_PML_WaveSolver(start_time)

    def RunForSteps(self, n: int) -> np.ndarray:
        return self.GetSolver().step(n)

    def Run(self, n_steps: Optional[int] = None, audio_path: Optional[str] = None, chunk: int = 1000) -> np.ndarray:
        """Step `n_steps` (default scene.steps) and append the listener rows to
        `audio_path` (all_audio.dat layout: raw doubles, step-major)."""
        n = int(n_steps if n_steps is not None else self.scene.steps)
        rows = []
        done = 0
        while done < n:
            m = min(chunk, n - done)
            y = self.GetSolver().step(m)
            if audio_path:
                write_audio(audio_path, y)
            rows.append(y)
            done += m
        return np.concatenate(rows, axis=0) if rows else np.zeros((0, self.scene.n_listeners))


def write_audio(path: str, rows: np.ndarray):
    data = np.ascontiguousarray(rows, dtype=np.float64)
    check(load().fdtd_audio_append(path.encode(), data.ctypes.data, data.size))


def device_count() -> int:
    n = C.c_int32(0)
    st = load().fdtd_device_count(C.byref(n))
    return int(n.value) if st == 0 else 0


def write_matrix(path: str, a) -> None:
    """IO::writeMatrixX<double>(a, path, IO::BINARY): int32 rows, int32 cols, row-major doubles."""
    a = np.ascontiguousarray(np.atleast_2d(np.asarray(a, dtype=np.float64)))
    check(load().fdtd_matrix_write(path.encode(), a.shape[0], a.shape[1], a.ctypes.data))


def read_matrix(path: str) -> np.ndarray:
    """MATRIX::read / the reader of write_matrix: a (rows, cols) array."""
    L = load()
    r, c = C.c_int32(0), C.c_int32(0)
    check(L.fdtd_matrix_read(path.encode(), C.byref(r), C.byref(c), None, 0))
    out = np.zeros((r.value, c.value), dtype=np.float64)
    check(L.fdtd_matrix_read(path.encode(), C.byref(r), C.byref(c), out.ctypes.data, out.size))
    return out


def read_obj(path: str, scale: float = 1.0):
    """Wavefront .obj surface mesh as a TriangleMesh (the library's reader:
    "v" and "f" records, polygons fanned, coordinates times `scale`)."""
    from .scene import TriangleMesh
    L = load()
    nv, nt = C.c_int32(0), C.c_int32(0)
    check(L.fdtd_read_obj(str(path).encode(), float(scale), C.byref(nv), C.byref(nt), None, None))
    v = np.zeros((nv.value, 3), dtype=np.float64)
    t = np.zeros((nt.value, 3), dtype=np.int32)
    check(L.fdtd_read_obj(str(path).encode(), float(scale), C.byref(nv), C.byref(nt), v.ctypes.data, t.ctypes.data))
    return TriangleMesh(v, t)
