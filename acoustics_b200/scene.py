"""Scene description mirrored from include/fdtd_c.h, and the seeded synthetic
scenes of the benchmark workloads.

The reference builds the same information from its XML scene through
ImpulseResponseParser (src/parser/ImpulseResponseParser.cpp:55-751):
`<solver>` settings, `<solver_control_policy type="static">`, rigid objects,
`<gaussian_pressure_source>` and `<listening_point_list>`.  Objects are analytic
primitives standing in for FDTD_RigidObject meshes; their boundary
acceleration replaces the vibrational sources of
FDTD_RigidObject::EvaluateBoundaryAcceleration (FDTD_RigidObject.cpp:330-368).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

SHAPE_SPHERE, SHAPE_BOX, SHAPE_ELLIPSOID, SHAPE_MESH = 0, 1, 2, 3
ACCEL_NONE, ACCEL_GAUSSIAN_TRANSLATION, ACCEL_GAUSSIAN_PULSATION = 0, 1, 2
MOTION_STATIC, MOTION_BALLISTIC, MOTION_KEYFRAMED = 0, 1, 2
PRECISION_FP64, PRECISION_FP32_COMPENSATED = 0, 1
KERNEL_FUSED, KERNEL_PHASED = 0, 1
PML_STATE_AUTO, PML_STATE_FULL = 0, 1
SHELL_STAGING_AUTO, SHELL_STAGING_RING, SHELL_STAGING_TMA = 0, 1, 2
BOUNDARY_RASTERIZE, BOUNDARY_FULLY_COUPLED = 0, 1

CELL_BULK, CELL_GHOST, CELL_VALID_HISTORY, CELL_PML, CELL_CONSTRAINT = 1, 2, 4, 8, 16
(FIELD_PRESSURE, FIELD_PRESSURE_PREV, FIELD_PML_PX, FIELD_PML_PY, FIELD_PML_PZ,
 FIELD_VX, FIELD_VY, FIELD_VZ) = range(8)

STATUS = {
    0: "FDTD_OK", 1: "FDTD_END_OF_TIME", -1: "FDTD_ERR_INVALID_ARG", -2: "FDTD_ERR_OOM",
    -3: "FDTD_ERR_CUDA", -4: "FDTD_ERR_NUMERIC", -5: "FDTD_ERR_TIMEOUT",
    -6: "FDTD_ERR_GEOMETRY", -7: "FDTD_ERR_UNSUPPORTED", -8: "FDTD_ERR_IO", -9: "FDTD_ERR_BUSY",
    -10: "FDTD_ERR_CANCELLED",
}
STATUS_CODE = {name: code for code, name in STATUS.items()}


class ObjectDesc(C.Structure):
    _fields_ = [
        ("shape", C.c_int32), ("accel_kind", C.c_int32), ("motion", C.c_int32), ("mesh", C.c_int32),
        ("center", C.c_double * 3), ("rotation", C.c_double * 9), ("size", C.c_double * 3),
        ("accel_amplitude", C.c_double), ("accel_t0", C.c_double), ("accel_tau", C.c_double),
        ("accel_dir", C.c_double * 3), ("velocity", C.c_double * 3), ("gravity", C.c_double * 3),
    ]


class PlaneDesc(C.Structure):
    _fields_ = [("normal_dir", C.c_int32), ("normal_sign", C.c_int32), ("height", C.c_double)]


class GaussianSourceDesc(C.Structure):
    _fields_ = [
        ("position", C.c_double * 3), ("width_time", C.c_double), ("width_space", C.c_double),
        ("offset_time", C.c_double), ("normalize_constant", C.c_double),
    ]


class MeshDesc(C.Structure):
    _fields_ = [("n_vertices", C.c_int32), ("n_triangles", C.c_int32),
                ("vertices", C.POINTER(C.c_double)), ("triangles", C.POINTER(C.c_int32))]


class KeyframeTrackDesc(C.Structure):
    _fields_ = [("object", C.c_int32), ("n_frames", C.c_int32), ("step", C.c_double),
                ("frames", C.POINTER(C.c_double))]


class SceneDesc(C.Structure):
    _fields_ = [
        ("cell_size", C.c_double), ("divisions", C.c_int32 * 3),
        ("boundary_condition_preset", C.c_int32), ("domain_center", C.c_double * 3),
        ("sound_speed", C.c_double), ("density", C.c_double), ("time_step", C.c_double),
        ("pml_width", C.c_double), ("pml_strength", C.c_double),
        ("air_viscosity_alpha", C.c_double), ("start_time", C.c_double), ("end_time", C.c_double),
        ("n_objects", C.c_int32), ("n_constraints", C.c_int32), ("n_sources", C.c_int32),
        ("n_listeners", C.c_int32),
        ("objects", C.POINTER(ObjectDesc)), ("constraints", C.POINTER(PlaneDesc)),
        ("sources", C.POINTER(GaussianSourceDesc)), ("listeners", C.POINTER(C.c_double)),
        ("boundary_handling", C.c_int32), ("n_meshes", C.c_int32), ("meshes", C.POINTER(MeshDesc)),
        ("n_tracks", C.c_int32), ("tracks", C.POINTER(KeyframeTrackDesc)),
    ]


class Options(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("device", C.c_int32), ("kernel", C.c_int32),
        ("graph_steps", C.c_int32), ("tile_y", C.c_int32), ("x_chunk", C.c_int32),
        ("pml_state", C.c_int32), ("shell_staging", C.c_int32),
    ]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("max_members", C.c_int32), ("chunk_steps", C.c_int32),
                ("preempt", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("submitted", "completed", "failed", "queued", "running", "peak_members",
                                         "peak_device_bytes")] + \
               [(n, C.c_double) for n in ("p50_latency_s", "p99_latency_s", "mean_latency_s", "span_s",
                                          "solves_per_s", "cell_steps_per_s")] + \
               [(n, C.c_int64) for n in ("device_bytes_in_use", "cancelled", "evictions")]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = 0, 1, 2, 3, 4


class SolverInfo(C.Structure):
    _fields_ = [
        ("divisions", C.c_int32 * 3), ("n_listeners", C.c_int32), ("n_cells", C.c_int64),
        ("n_pml_cells", C.c_int64), ("n_interior_cells", C.c_int64), ("device_bytes", C.c_int64),
        ("step_index", C.c_int64), ("time", C.c_double), ("time_step", C.c_double),
        ("algorithmic_bytes_per_step", C.c_double),
    ]


class GhostFace(C.Structure):
    _fields_ = [
        ("owner_cell", C.c_int32), ("neighbour_cell", C.c_int32), ("topology", C.c_int32),
        ("type", C.c_int32), ("boundary_object", C.c_int32), ("_pad", C.c_int32),
        ("key", C.c_uint64),
    ]


# fdtd_cell: MAC_Grid::Cell as GetCell fills it (MAC_Grid.h:187-215)
CELL_DTYPE = np.dtype([
    ("index", "<i4"), ("indices", "<i4", (3,)), ("flags", "<i4"), ("n_gc_value", "<i4"),
    ("r_identity", "<f8"), ("centroid", "<f8", (3,)), ("lower_corner", "<f8", (3,)),
    ("upper_corner", "<f8", (3,)), ("gc_value", "<f8", (6,)), ("p_directional", "<f8", (3,)),
    ("p_full", "<f8"), ("vx", "<f8", (2,)), ("vy", "<f8", (2,)), ("vz", "<f8", (2,)), ("h", "<f8"),
    ("laplacian", "<f8"),
])
CELLINFO_LAPLACIAN, CELLINFO_PML_STATE = 1 << 8, 1 << 9

GHOST_FACE_DTYPE = np.dtype([
    ("owner_cell", "<i4"), ("neighbour_cell", "<i4"), ("topology", "<i4"), ("type", "<i4"),
    ("boundary_object", "<i4"), ("_pad", "<i4"), ("key", "<u8"),
])


@dataclass
class RigidObject:
    """An analytic FDTD_RigidObject: shape, pose, boundary acceleration, motion."""
    shape: int
    center: Sequence[float]
    size: Sequence[float]
    rotation: Sequence[float] = (1, 0, 0, 0, 1, 0, 0, 0, 1)
    accel_kind: int = ACCEL_NONE
    accel_amplitude: float = 0.0
    accel_t0: float = 0.0
    accel_tau: float = 1.0
    accel_dir: Sequence[float] = (0.0, 0.0, 1.0)
    motion: int = MOTION_STATIC
    velocity: Sequence[float] = (0.0, 0.0, 0.0)
    gravity: Sequence[float] = (0.0, 0.0, 0.0)
    mesh: int = 0  # SHAPE_MESH: index into Scene.meshes


@dataclass
class TriangleMesh:
    """Closed triangle mesh in its object frame (world = rotation @ v + center),
    counter-clockwise from outside; see fdtd_mesh_desc."""
    vertices: np.ndarray   # (n, 3) float64
    triangles: np.ndarray  # (m, 3) int32


@dataclass
class KeyframeTrack:
    """Keyframes of a MOTION_KEYFRAMED object (see fdtd_keyframe_track): frame i at
    time i * step, frames[i] = (cx, cy, cz, qw, qx, qy, qz)."""
    object: int
    step: float
    frames: np.ndarray  # (n, 7) float64


@dataclass
class PlaneConstraint:
    normal_dir: int
    normal_sign: int
    height: float


@dataclass
class GaussianSource:
    position: Sequence[float]
    width_time: float
    width_space: float = 0.0          # <= 0 -> sound_speed * width_time
    offset_time: float = 0.0
    normalize_constant: float = 0.0   # 0 -> 1/(sqrt(2 pi) width_space)^3


@dataclass
class Scene:
    """Solver settings + scene; field names follow PML_WaveSolver_Settings
    (src/wavesolver/PML_WaveSolver_Settings.h:17-99)."""
    cell_size: float
    divisions: Sequence[int]
    time_step: float
    domain_center: Sequence[float] = (0.0, 0.0, 0.0)
    sound_speed: float = 343.0
    density: float = 1.184
    pml_width: float = 10.0
    pml_strength: float = 1.0e6
    boundary_condition_preset: int = 0
    air_viscosity_alpha: float = 0.0
    boundary_handling: int = 0  # BOUNDARY_RASTERIZE / BOUNDARY_FULLY_COUPLED
    start_time: float = 0.0
    end_time: float = 0.0
    objects: List[RigidObject] = field(default_factory=list)
    constraints: List[PlaneConstraint] = field(default_factory=list)
    sources: List[GaussianSource] = field(default_factory=list)
    listeners: Optional[np.ndarray] = None
    meshes: List[TriangleMesh] = field(default_factory=list)
    tracks: List[KeyframeTrack] = field(default_factory=list)
    steps: int = 0
    name: str = "scene"

    @property
    def n_cells(self) -> int:
        return int(self.divisions[0]) * int(self.divisions[1]) * int(self.divisions[2])

    @property
    def n_listeners(self) -> int:
        return 0 if self.listeners is None else int(np.asarray(self.listeners).reshape(-1, 3).shape[0])

    def to_c(self):
        """Return (SceneDesc, keepalive) — keepalive holds the arrays the struct points to."""
        objs = (ObjectDesc * max(1, len(self.objects)))()
        for i, o in enumerate(self.objects):
            d = objs[i]
            d.shape, d.accel_kind, d.motion = int(o.shape), int(o.accel_kind), int(o.motion)
            d.mesh = int(o.mesh)
            d.center[:] = [float(x) for x in o.center]
            d.rotation[:] = [float(x) for x in o.rotation]
            sz = list(o.size) + [0.0] * (3 - len(o.size))
            d.size[:] = [float(x) for x in sz[:3]]
            d.accel_amplitude, d.accel_t0, d.accel_tau = o.accel_amplitude, o.accel_t0, o.accel_tau
            d.accel_dir[:] = [float(x) for x in o.accel_dir]
            d.velocity[:] = [float(x) for x in o.velocity]
            d.gravity[:] = [float(x) for x in o.gravity]
        planes = (PlaneDesc * max(1, len(self.constraints)))()
        for i, p in enumerate(self.constraints):
            planes[i].normal_dir, planes[i].normal_sign, planes[i].height = p.normal_dir, p.normal_sign, p.height
        srcs = (GaussianSourceDesc * max(1, len(self.sources)))()
        for i, s in enumerate(self.sources):
            srcs[i].position[:] = [float(x) for x in s.position]
            srcs[i].width_time = s.width_time
            srcs[i].width_space = s.width_space
            srcs[i].offset_time = s.offset_time
            srcs[i].normalize_constant = s.normalize_constant
        mesh_arrays = []
        meshes = (MeshDesc * max(1, len(self.meshes)))()
        for i, m in enumerate(self.meshes):
            v = np.ascontiguousarray(np.asarray(m.vertices, dtype=np.float64).reshape(-1, 3))
            t = np.ascontiguousarray(np.asarray(m.triangles, dtype=np.int32).reshape(-1, 3))
            mesh_arrays += [v, t]
            meshes[i].n_vertices, meshes[i].n_triangles = v.shape[0], t.shape[0]
            meshes[i].vertices = v.ctypes.data_as(C.POINTER(C.c_double))
            meshes[i].triangles = t.ctypes.data_as(C.POINTER(C.c_int32))
        track_arrays = []
        tracks = (KeyframeTrackDesc * max(1, len(self.tracks)))()
        for i, t in enumerate(self.tracks):
            f = np.ascontiguousarray(np.asarray(t.frames, dtype=np.float64).reshape(-1, 7))
            track_arrays.append(f)
            tracks[i].object, tracks[i].n_frames, tracks[i].step = int(t.object), f.shape[0], float(t.step)
            tracks[i].frames = f.ctypes.data_as(C.POINTER(C.c_double))
        L = self.n_listeners
        lis = np.ascontiguousarray(np.asarray(self.listeners if L else np.zeros((1, 3)), dtype=np.float64).reshape(-1))
        desc = SceneDesc()
        desc.cell_size = self.cell_size
        desc.divisions[:] = [int(x) for x in self.divisions]
        desc.boundary_condition_preset = self.boundary_condition_preset
        desc.boundary_handling = int(self.boundary_handling)
        desc.domain_center[:] = [float(x) for x in self.domain_center]
        desc.sound_speed, desc.density, desc.time_step = self.sound_speed, self.density, self.time_step
        desc.pml_width, desc.pml_strength = self.pml_width, self.pml_strength
        desc.air_viscosity_alpha = self.air_viscosity_alpha
        desc.start_time, desc.end_time = self.start_time, self.end_time
        desc.n_objects, desc.n_constraints = len(self.objects), len(self.constraints)
        desc.n_sources, desc.n_listeners = len(self.sources), L
        desc.objects = C.cast(objs, C.POINTER(ObjectDesc))
        desc.constraints = C.cast(planes, C.POINTER(PlaneDesc))
        desc.sources = C.cast(srcs, C.POINTER(GaussianSourceDesc))
        desc.listeners = lis.ctypes.data_as(C.POINTER(C.c_double))
        desc.n_meshes = len(self.meshes)
        desc.meshes = C.cast(meshes, C.POINTER(MeshDesc))
        desc.n_tracks = len(self.tracks)
        desc.tracks = C.cast(tracks, C.POINTER(KeyframeTrackDesc))
        return desc, (objs, planes, srcs, lis, meshes, mesh_arrays, tracks, track_arrays)

    # ---- geometry helpers (BoundingBox.h:89-99, ScalarField.cpp:29-50) ----
    def bbox(self):
        h = self.cell_size
        mn = np.array([self.domain_center[d] - h * float(self.divisions[d]) / 2.0 for d in range(3)])
        return mn, mn + h * np.asarray(self.divisions, dtype=np.float64)

    def algorithmic_words_per_step(self) -> int:
        """3 words per non-PML cell + 14 per PML cell."""
        n_pml = self.n_pml_cells()
        return 3 * (self.n_cells - n_pml) + 14 * n_pml

    def n_pml_cells(self) -> int:
        h = self.cell_size
        w = self.pml_width * h + 1e-12
        mn, mx = self.bbox()
        masks = []
        for d in range(3):
            c = mn[d] + (0.5 + np.arange(self.divisions[d])) * h
            masks.append(((c - mn[d]) <= w) | ((mx[d] - c) <= w))
        inner = [int((~m).sum()) for m in masks]
        return self.n_cells - inner[0] * inner[1] * inner[2]


def icosphere(radius: float, level: int = 2) -> TriangleMesh:
    """Closed sphere mesh: an icosahedron with each triangle split into four
    `level` times, vertices on the sphere; counter-clockwise from outside."""
    g = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, g, 0), (1, g, 0), (-1, -g, 0), (1, -g, 0), (0, -1, g), (0, 1, g), (0, -1, -g), (0, 1, -g),
         (g, 0, -1), (g, 0, 1), (-g, 0, -1), (-g, 0, 1)]
    v = [np.asarray(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        mid = {}

        def m(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                p = v[a] + v[b]
                v.append(p / np.linalg.norm(p))
                mid[key] = len(v) - 1
            return mid[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    V = np.asarray(v) * radius
    T = np.asarray(f, dtype=np.int32)
    # outward orientation
    n = np.cross(V[T[:, 1]] - V[T[:, 0]], V[T[:, 2]] - V[T[:, 0]])
    flip = np.einsum("ij,ij->i", n, V[T].mean(axis=1)) < 0
    T[flip] = T[flip][:, ::-1]
    return TriangleMesh(V, T)


def box_mesh(half) -> TriangleMesh:
    """Closed box mesh with half extents `half`, two triangles per face,
    counter-clockwise from outside."""
    hx, hy, hz = [float(x) for x in half]
    V = np.array([[sx * hx, sy * hy, sz * hz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)])
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    T = []
    for a, b, c, d in quads:
        T += [(a, b, c), (a, c, d)]
    T = np.asarray(T, dtype=np.int32)
    n = np.cross(V[T[:, 1]] - V[T[:, 0]], V[T[:, 2]] - V[T[:, 0]])
    flip = np.einsum("ij,ij->i", n, V[T].mean(axis=1)) < 0
    T[flip] = T[flip][:, ::-1]
    return TriangleMesh(V, T)


def reference_time_step(h: float, c: float = 343.0) -> float:
    """k = 0.5 h / (c sqrt 3): the CFL-limited step of the configs."""
    return 0.5 * h / (c * math.sqrt(3.0))


def _non_pml_box(sc: Scene, margin_cells: float):
    mn, mx = sc.bbox()
    pad = (sc.pml_width + margin_cells) * sc.cell_size
    return mn + pad, mx - pad


def _sample_listeners(rng, sc: Scene, n: int, keep_out) -> np.ndarray:
    lo, hi = _non_pml_box(sc, 1.0)
    pts = []
    while len(pts) < n:
        p = rng.uniform(lo, hi)
        if all(f(p) for f in keep_out):
            pts.append(p)
    return np.asarray(pts, dtype=np.float64)


def config1(seed_src: int = 1, seed_lis: int = 2, divisions=(64, 64, 64), pml_width: float = 10,
            radius: float = 0.04, steps: int = 500) -> Scene:
    """64^3, h=5 mm, 10-cell PML, sphere r=4 cm at the centre, Gaussian pulse
    sigma_t=2e-4 s at a seeded offset outside the sphere, 8 listeners, 500 steps.
    Other grid sizes re-draw the source and listeners inside the new fluid region."""
    h = 0.005
    sc = Scene(cell_size=h, divisions=tuple(divisions), time_step=reference_time_step(h), pml_width=pml_width,
               steps=steps, name="cfg1_64cube_sphere_fp64" if tuple(divisions) == (64, 64, 64) else "cfg1_variant")
    r = radius
    sc.objects.append(RigidObject(SHAPE_SPHERE, (0.0, 0.0, 0.0), (r, 0, 0)))
    rng = np.random.default_rng(seed_src)
    lo, hi = _non_pml_box(sc, 2.0)
    while True:
        p = rng.uniform(lo, hi)
        if np.linalg.norm(p) > r + 3 * h:
            break
    sc.sources.append(GaussianSource(tuple(p), 2e-4))
    sc.listeners = _sample_listeners(np.random.default_rng(seed_lis), sc, 8,
                                     [lambda q: np.linalg.norm(q) > r + 2 * h])
    return sc


def config2(seed_pose: int = 3, seed_lis: int = 4, steps: int = 4000, n: int = 256) -> Scene:
    """256^3, h=2.5 mm, 16-cell PML, sphere r=3 cm + axis-aligned box 4x2x1 cm +
    ellipsoid 3/2/1 cm at seeded non-overlapping poses, Gaussian-in-time
    translational boundary acceleration of amplitude 1e3 m/s^2, 64 listeners on a
    seeded sphere shell.  n != 256 keeps the 64 cm domain and PML thickness with
    h = 0.64/n."""
    h = 0.0025 * 256 / n
    k = reference_time_step(h)
    sc = Scene(cell_size=h, divisions=(n, n, n), time_step=k, pml_width=16 * n / 256, steps=steps,
               name="cfg2_256cube_3objects" if n == 256 else f"cfg2_{n}cube_3objects")
    rng = np.random.default_rng(seed_pose)
    half_ext = [np.array([0.03, 0.03, 0.03]), np.array([0.02, 0.01, 0.005]), np.array([0.03, 0.02, 0.01])]
    lo, hi = _non_pml_box(sc, 12.0 * n / 256)
    centers = []
    while len(centers) < 3:
        e = half_ext[len(centers)]
        p = rng.uniform(lo + e, hi - e)
        if all(np.linalg.norm(p - q) > 0.075 for q in centers):
            centers.append(p)
    tau = 1.0e-4
    t0 = 4 * tau
    dirs = rng.normal(size=(3, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    shapes = [(SHAPE_SPHERE, (0.03, 0, 0)), (SHAPE_BOX, (0.02, 0.01, 0.005)), (SHAPE_ELLIPSOID, (0.03, 0.02, 0.01))]
    for i, (shp, size) in enumerate(shapes):
        sc.objects.append(RigidObject(shp, tuple(centers[i]), size, accel_kind=ACCEL_GAUSSIAN_TRANSLATION,
                                      accel_amplitude=1.0e3, accel_t0=t0, accel_tau=tau,
                                      accel_dir=tuple(dirs[i])))
    # 64 listeners on a seeded sphere shell around the domain centre
    rng = np.random.default_rng(seed_lis)
    lo, hi = _non_pml_box(sc, 2.0)
    R = 0.9 * float(np.min(hi - lo)) / 2.0
    pts = []
    while len(pts) < 64:
        v = rng.normal(size=3)
        p = v / np.linalg.norm(v) * R
        if all(np.linalg.norm(p - q) > 0.045 for q in centers):
            pts.append(p)
    sc.listeners = np.asarray(pts)
    return sc


def random_scene(rng, edge_lo: int, edge_hi: int, n_obj_max: int, n_listeners: int,
                 steps_lo: int, steps_hi: int, name: str, h: float = 0.005, pml: int = 8) -> Scene:
    """Uneven scene: per-axis edges log-uniform in [edge_lo, edge_hi], 1..n_obj_max
    spheres/boxes, one Gaussian source, listeners in the non-PML fluid."""
    dims = tuple(int(round(math.exp(rng.uniform(math.log(edge_lo), math.log(edge_hi))))) for _ in range(3))
    steps = int(rng.integers(steps_lo, steps_hi + 1))
    sc = Scene(cell_size=h, divisions=dims, time_step=reference_time_step(h), pml_width=pml, steps=steps,
               name=name)
    lo, hi = _non_pml_box(sc, 3.0)
    span = hi - lo
    nobj = int(rng.integers(1, n_obj_max + 1))
    placed = []
    for _ in range(nobj):
        for _try in range(50):
            rad = float(rng.uniform(2.0, max(2.5, min(6.0, 0.2 * span.min() / h)))) * h
            e = np.array([rad, rad, rad])
            if np.any(span <= 2 * e):
                break
            p = rng.uniform(lo + e, hi - e)
            if all(np.linalg.norm(p - q) > rad + r2 + 2 * h for q, r2 in placed):
                placed.append((p, rad))
                if rng.uniform() < 0.5:
                    sc.objects.append(RigidObject(SHAPE_SPHERE, tuple(p), (rad, 0, 0)))
                else:
                    sc.objects.append(RigidObject(SHAPE_BOX, tuple(p), (rad, 0.7 * rad, 0.5 * rad)))
                break
    keep = [lambda q, placed=placed: all(np.linalg.norm(q - p) > r + 2 * h for p, r in placed)]
    src = _sample_listeners(rng, sc, 1, keep)[0]
    sc.sources.append(GaussianSource(tuple(src), 1e-4))
    sc.listeners = _sample_listeners(rng, sc, n_listeners, keep)
    return sc


def config3(seed: int = 5, n_scenes: int = 64) -> List[Scene]:
    """64 uneven scenes, edges log-uniform in [48,160] per axis, 1000-3000 steps,
    1-3 spheres/boxes each."""
    rng = np.random.default_rng(seed)
    return [random_scene(rng, 48, 160, 3, 8, 1000, 3000, f"cfg3_scene{i}") for i in range(n_scenes)]


def config4(seed: int = 9, n_requests: int = 16, rate_per_s: float = 2.0):
    """Serving stream: Poisson arrivals at `rate_per_s` (seeded), each request a scene
    with grid edges log-uniform in [64, 256], 1000-8000 steps, 1-4 rigid
    spheres/boxes, a random source and 16 listeners.  Returns [(arrival_s, Scene)]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += float(rng.exponential(1.0 / rate_per_s))
        out.append((t, random_scene(rng, 64, 256, 4, 16, 1000, 8000, f"cfg4_req{i}")))
    return out


def config5(seed: int = 7, steps: int = 6000) -> Scene:
    """384x384x256, h=2 mm, two spheres r=2.5 cm on seeded ballistic paths that
    meet mid-run, a Gaussian pulse to scatter, 32 listeners; PML width 10."""
    h = 0.002
    k = reference_time_step(h)
    sc = Scene(cell_size=h, divisions=(384, 384, 256), time_step=k, pml_width=10, steps=steps,
               name="cfg5_384x384x256_moving")
    rng = np.random.default_rng(seed)
    T = steps * k
    r = 0.025
    meet = rng.uniform(-0.02, 0.02, size=3)
    g = np.array([0.0, 0.0, -9.81])
    off = np.array([0.12, 0.0, 0.0]) + rng.uniform(-0.01, 0.01, size=3)
    for sgn in (+1, -1):
        # x(T/2) = meet +- (r + small gap): choose v0 so that they touch at T/2
        x_half = meet + sgn * np.array([r, 0, 0])
        x0 = meet + sgn * off
        v0 = (x_half - x0 - 0.5 * g * (T / 2) ** 2) / (T / 2)
        sc.objects.append(RigidObject(SHAPE_SPHERE, tuple(x0), (r, 0, 0), motion=MOTION_BALLISTIC,
                                      velocity=tuple(v0), gravity=tuple(g)))
    sc.sources.append(GaussianSource((0.0, 0.12, 0.0), 1e-4))
    # the run ends after `steps` steps (<time_end>): the library can then check
    # that the spheres stay clear of the PML throughout
    sc.end_time = steps * k
    lis = []
    rng2 = np.random.default_rng(seed + 100)
    lo, hi = _non_pml_box(sc, 2.0)
    while len(lis) < 32:
        p = rng2.uniform(lo, hi)
        if abs(p[1]) > 0.06 or abs(p[2]) > 0.06:
            lis.append(p)
    sc.listeners = np.asarray(lis)
    return sc


def scaled(sc: Scene, divisions: Sequence[int], steps: Optional[int] = None) -> Scene:
    """A copy of `sc` with another grid resolution (same cell size)."""
    import copy
    s2 = copy.deepcopy(sc)
    s2.divisions = tuple(int(x) for x in divisions)
    if steps is not None:
        s2.steps = steps
    return s2
