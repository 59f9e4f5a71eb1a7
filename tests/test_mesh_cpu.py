"""Triangle-mesh bodies without a GPU: the .obj reader, mesh validation at the
C-ABI (closed, consistently oriented surfaces only, as the reference's signed
distance field requires), the <rigid_object> XML element, and the oracle's mesh
queries against the analytic sphere they approximate."""
import ctypes as C

import numpy as np
import pytest

from acoustics_b200 import scene as S
from tests._util import small_scene_with


OBJ_TEXT = """# unit cube, quads, mixed index forms
v -0.5 -0.5 -0.5
v 0.5 -0.5 -0.5
v 0.5 0.5 -0.5
v -0.5 0.5 -0.5
v -0.5 -0.5 0.5
v 0.5 -0.5 0.5
v 0.5 0.5 0.5
v -0.5 0.5 0.5
vn 0 0 1
f 1 4 3 2
f 5/1 6/1 7/1 8/1
f 1//1 2//1 6//1 5//1
f 2 3 7 6
f 3 4 8 7
f -8 -4 -1 -5
"""


def test_read_obj_fans_polygons_and_scales(fdtd_lib, tmp_path):
    from acoustics_b200.solver import read_obj
    p = tmp_path / "cube.obj"
    p.write_text(OBJ_TEXT)
    m = read_obj(str(p), scale=0.02)
    assert m.vertices.shape == (8, 3) and m.triangles.shape == (12, 3)
    assert np.allclose(np.abs(m.vertices), 0.01)
    assert list(m.triangles[0]) == [0, 3, 2] and list(m.triangles[1]) == [0, 2, 1]
    assert list(m.triangles[-2]) == [0, 4, 7] and list(m.triangles[-1]) == [0, 7, 3]
    # the cube is closed and consistently oriented: a scene with it is valid
    sc = small_scene_with(S.RigidObject(S.SHAPE_MESH, (0.0, 0.0, 0.0), (0, 0, 0), mesh=0), meshes=[m])
    from acoustics_b200.batch import scene_info
    info = scene_info(sc)
    assert info.device_bytes > 0


def _status_of(fdtd_lib, sc):
    from acoustics_b200.scene import Options, SolverInfo
    desc, keep = sc.to_c()
    info = SolverInfo()
    st = fdtd_lib.fdtd_scene_info(C.byref(desc), C.byref(Options()), C.byref(info))
    del keep
    return st


@pytest.mark.parametrize("defect", ["open", "flipped", "index", "degenerate"])
def test_invalid_meshes_are_rejected(fdtd_lib, defect):
    m = S.icosphere(0.02, 1)
    T = m.triangles.copy()
    if defect == "open":
        T = T[1:]
    elif defect == "flipped":
        T[0] = T[0][::-1]
    elif defect == "index":
        T[0, 0] = len(m.vertices)
    else:
        T[0, 1] = T[0, 0]
    sc = small_scene_with(S.RigidObject(S.SHAPE_MESH, (0.0, 0.0, 0.0), (0, 0, 0), mesh=0),
                          meshes=[S.TriangleMesh(m.vertices, T)])
    st = _status_of(fdtd_lib, sc)
    assert st in (S.STATUS_CODE["FDTD_ERR_GEOMETRY"], S.STATUS_CODE["FDTD_ERR_INVALID_ARG"])
    assert fdtd_lib.fdtd_last_error()


def test_mesh_index_checked(fdtd_lib):
    m = S.icosphere(0.02, 1)
    sc = small_scene_with(S.RigidObject(S.SHAPE_MESH, (0.0, 0.0, 0.0), (0, 0, 0), mesh=1), meshes=[m])
    assert _status_of(fdtd_lib, sc) == S.STATUS_CODE["FDTD_ERR_INVALID_ARG"]
    sc = small_scene_with(S.RigidObject(S.SHAPE_MESH, (0.0, 0.0, 0.0), (0, 0, 0), mesh=0), meshes=[m])
    sc.boundary_handling = S.BOUNDARY_FULLY_COUPLED  # mesh bodies take the coupled rows too
    assert _status_of(fdtd_lib, sc) == S.STATUS_CODE["FDTD_OK"]
    sc = small_scene_with(S.RigidObject(S.SHAPE_MESH, (0.0, 0.0, 0.0), (0, 0, 0), mesh=0,
                                        accel_kind=S.ACCEL_GAUSSIAN_PULSATION, accel_amplitude=1.0,
                                        accel_tau=1e-4), meshes=[m])
    assert _status_of(fdtd_lib, sc) == S.STATUS_CODE["FDTD_ERR_UNSUPPORTED"]


XML = """<?xml version="1.0" ?>
<impulse_response>
  <solver sound_speed="343" density="1.184" cellsize="0.005" stop_time="0.001" number_of_timesteps="20"
          timestepfrequency="237635.4" output_pattern="out/%s" write_pressure_field_to_disk="0"
          PML_width="6" PML_strength="1000000.0"/>
  <solver_control_policy type="static" gridresolution="40"/>
  <scene>
    <rigid_object working_directory="meshes" object_prefix="cube" id="0" fieldresolution="64" scale="0.04"
                  initial_position_x="0.01" initial_position_y="0.0" initial_position_z="-0.005"/>
  </scene>
  <pressure_source>
    <gaussian_pressure_source source_width_time="2e-4" source_position_x="0.0" source_position_y="0.05"
                              source_position_z="0.0"/>
  </pressure_source>
  <listening_point_list>
    <listening_point x="0.0" y="-0.05" z="0.0"/>
  </listening_point_list>
</impulse_response>
"""


def test_xml_rigid_object_reads_the_mesh(fdtd_lib, tmp_path):
    """<rigid_object working_directory= object_prefix= scale= initial_position_*=>
    (ImpulseResponseParser.cpp:210-219): the .obj is read (relative to the XML
    file here) and scaled, the initial position is the object's centre."""
    from acoustics_b200.solver import scene_from_xml
    (tmp_path / "meshes").mkdir()
    (tmp_path / "meshes" / "cube.obj").write_text(OBJ_TEXT)
    p = tmp_path / "scene.xml"
    p.write_text(XML)
    sc = scene_from_xml(str(p))
    assert len(sc.objects) == 1 and sc.objects[0].shape == S.SHAPE_MESH and sc.objects[0].mesh == 0
    assert tuple(sc.objects[0].center) == (0.01, 0.0, -0.005)
    assert len(sc.meshes) == 1 and sc.meshes[0].triangles.shape == (12, 3)
    assert np.allclose(np.abs(sc.meshes[0].vertices), 0.02)
    # a missing mesh file is an I/O error
    p.write_text(XML.replace('object_prefix="cube"', 'object_prefix="nothing"'))
    h = C.c_void_p()
    assert fdtd_lib.fdtd_scene_from_xml(str(p).encode(), C.byref(h)) == S.STATUS_CODE["FDTD_ERR_IO"]


def test_oracle_mesh_sphere_close_to_analytic(oracle_lib):
    """The oracle's mesh queries on an icosphere inscribed in a sphere: the two
    classifications differ only in a thin shell at the surface."""
    def mk(mesh):
        sc = S.Scene(cell_size=0.005, divisions=(40, 40, 40), time_step=S.reference_time_step(0.005),
                     pml_width=6, steps=10)
        if mesh:
            sc.meshes.append(S.icosphere(0.04, 3))
            sc.objects.append(S.RigidObject(S.SHAPE_MESH, (0.003, -0.002, 0.001), (0, 0, 0), mesh=0))
        else:
            sc.objects.append(S.RigidObject(S.SHAPE_SPHERE, (0.003, -0.002, 0.001), (0.04, 0, 0)))
        sc.sources.append(S.GaussianSource((0.0, 0.06, 0.0), 1e-4))
        sc.listeners = np.array([[0.0, -0.06, 0.01]])
        return sc
    fa, _ = oracle_lib.OracleSolver(mk(False)).classification()
    fm, _ = oracle_lib.OracleSolver(mk(True)).classification()
    solid_a = (fa & S.CELL_BULK) == 0
    solid_m = (fm & S.CELL_BULK) == 0
    assert solid_m.sum() > 0.97 * solid_a.sum()
    # the icosphere lies inside the sphere: it is never solid where the sphere is not
    assert not np.any(solid_m & ~solid_a)
    assert (solid_a != solid_m).sum() < 0.02 * solid_a.sum()


def _mesh_desc(m):
    v = np.ascontiguousarray(np.asarray(m.vertices, dtype=np.float64).reshape(-1, 3))
    t = np.ascontiguousarray(np.asarray(m.triangles, dtype=np.int32).reshape(-1, 3))
    d = S.MeshDesc()
    d.n_vertices, d.n_triangles = v.shape[0], t.shape[0]
    d.vertices = v.ctypes.data_as(C.POINTER(C.c_double))
    d.triangles = t.ctypes.data_as(C.POINTER(C.c_int32))
    return d, (v, t)


@pytest.mark.parametrize("shape", ["icosphere", "box"])
def test_mesh_distance_hierarchy_equals_brute_force(fdtd_lib, oracle_lib, shape):
    """The library's hierarchy walk (pruning, nearer child first, ties to the
    lowest triangle index) returns the oracle's every-triangle scan bit for bit:
    random points around the body, its vertices and its edge midpoints."""
    from oracle.loader import lib as olib
    m = S.icosphere(0.03, 3) if shape == "icosphere" else S.box_mesh((0.02, 0.011, 0.015))
    rng = np.random.default_rng(3)
    ext = np.abs(m.vertices).max(axis=0)
    pts = [rng.uniform(-1.6 * ext, 1.6 * ext, size=(20000, 3)), m.vertices,
           0.5 * (m.vertices[m.triangles[:, 0]] + m.vertices[m.triangles[:, 1]])]
    pts = np.ascontiguousarray(np.concatenate(pts))
    desc, keep = _mesh_desc(m)
    a = np.zeros(len(pts))
    b = np.zeros(len(pts))
    assert fdtd_lib.fdtd_mesh_signed_distance(C.byref(desc), len(pts), pts.ctypes.data, a.ctypes.data) == 0
    assert olib().oracle_mesh_sdf(C.byref(desc), len(pts), pts.ctypes.data, b.ctypes.data) == 0
    assert np.array_equal(a, b)
    if shape == "icosphere":  # inscribed polyhedron: within the facet depth of the sphere's distance
        r = np.linalg.norm(pts[:20000], axis=1) - 0.03
        assert np.all(np.abs(a[:20000] - r) < 0.03 * 0.01)
        assert np.all(np.sign(a[:20000][np.abs(r) > 1e-3]) == np.sign(r[np.abs(r) > 1e-3]))
    else:  # a box mesh is exact: the analytic box distance
        half = np.array([0.02, 0.011, 0.015])
        q = np.abs(pts[:20000]) - half
        out = np.linalg.norm(np.maximum(q, 0.0), axis=1)
        inn = np.minimum(q.max(axis=1), 0.0)
        assert np.allclose(a[:20000], out + inn, rtol=0, atol=1e-15)


def l_prism(scale=0.01):
    """Closed extruded L (the union of the boxes [0,2]x[0,1]x[0,1] and
    [0,1]x[0,2]x[0,1], times `scale`): a body with concave edges and vertices."""
    poly = [(0, 0), (2, 0), (2, 1), (1, 1), (1, 2), (0, 2)]  # counter-clockwise from +z
    n = len(poly)
    V = [(x, y, 0.0) for x, y in poly] + [(x, y, 1.0) for x, y in poly]
    T = []
    for a, b, c in [(0, 1, 2), (0, 2, 3), (0, 3, 4), (0, 4, 5)]:  # star-shaped from vertex 0
        T.append((n + a, n + b, n + c))  # top, normal +z
        T.append((a, c, b))              # bottom, normal -z
    for i in range(n):
        j = (i + 1) % n
        T += [(i, j, n + j), (i, n + j, n + i)]
    return S.TriangleMesh(np.asarray(V) * scale, np.asarray(T, dtype=np.int32))


def test_concave_mesh_signs_and_distances(fdtd_lib, oracle_lib):
    """Signs at concave edges and vertices (pseudo-normals), and exterior
    distances, against the L's closed form; library and oracle equal."""
    from oracle.loader import lib as olib
    m = l_prism(0.01)
    rng = np.random.default_rng(4)
    p = np.ascontiguousarray(rng.uniform(-0.01, 0.03, size=(40000, 3)))
    desc, keep = _mesh_desc(m)
    a = np.zeros(len(p))
    b = np.zeros(len(p))
    assert fdtd_lib.fdtd_mesh_signed_distance(C.byref(desc), len(p), p.ctypes.data, a.ctypes.data) == 0
    assert olib().oracle_mesh_sdf(C.byref(desc), len(p), p.ctypes.data, b.ctypes.data) == 0
    assert np.array_equal(a, b)

    def box_dist(q, lo, hi):
        d = np.maximum(np.maximum(lo - q, q - hi), 0.0)
        return np.linalg.norm(d, axis=1)
    d1 = box_dist(p, np.array([0, 0, 0.0]), np.array([0.02, 0.01, 0.01]))
    d2 = box_dist(p, np.array([0, 0, 0.0]), np.array([0.01, 0.02, 0.01]))
    inside = (d1 == 0) | (d2 == 0)
    outside = np.minimum(d1, d2)
    clear = (outside > 1e-9) | inside
    assert np.all(a[inside & (np.abs(a) > 1e-12)] < 0)
    assert np.all(a[~inside] > 0)
    assert np.allclose(a[~inside & clear], outside[~inside & clear], rtol=0, atol=1e-15)


def test_xml_mesh_scene_runs_in_the_oracle(fdtd_lib, oracle_lib, tmp_path):
    """A scene file with a <rigid_object> loads into the same scene the Python
    API builds, and the checker solves it: the cube is solid where it stands."""
    from acoustics_b200.solver import scene_from_xml
    (tmp_path / "meshes").mkdir()
    (tmp_path / "meshes" / "cube.obj").write_text(OBJ_TEXT)
    p = tmp_path / "scene.xml"
    p.write_text(XML)
    sc = scene_from_xml(str(p))
    sc.steps = 10
    o = oracle_lib.OracleSolver(sc)
    y = o.step(10)
    flags, faces = o.classification()
    assert y.shape == (10, 1) and np.all(np.isfinite(y))
    solid = (flags & S.CELL_BULK) == 0
    # a 4 cm cube at h = 5 mm: 8^3 cell centres inside, give or take the h/4 probes
    assert 8 ** 3 <= solid.sum() <= 10 ** 3
    assert len(faces) > 0
