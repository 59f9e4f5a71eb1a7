"""The reference project's own scene and mesh fixtures through the library's
readers (host only; skipped where the reference tree is absent):

* src/wavesolver/config_examples/config.xml names, one after the other, the
  features outside this path (modal transfer shaders, modal sound objects,
  object-file sequences, time-parallel chunking) and, with those removed,
  reads into a scene whose PML width the solver rejects as the Engquist path;
* work/meshes/ball_plane_scene/test_FDTD_RigidObject.xml lacks the
  <solver_control_policy> the reference's parser requires (ImpulseResponseParser.cpp:607);
  in the current schema, with the fixture mesh, it reads and the oracle steps it;
* the fixture meshes (small_ball, ball, bowl) are closed and consistently
  oriented; small_ball's committed copy (tests/golden/small_ball_mesh.npz)
  equals the file.
"""
import os
import re

import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200._lib import FDTDError

REF = "/root/reference"
pytestmark = pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
UNSUP, INVAL = S.STATUS_CODE["FDTD_ERR_UNSUPPORTED"], S.STATUS_CODE["FDTD_ERR_INVALID_ARG"]


def _read(path):
    from acoustics_b200.solver import scene_from_xml
    return scene_from_xml(str(path))


def _strip(text, element):
    """Remove every <element .../> or <element>...</element> from an XML text."""
    text = re.sub(r"<%s\b[^>]*/>" % element, "", text, flags=re.S)
    return re.sub(r"<%s\b.*?</%s>" % (element, element), "", text, flags=re.S)


def test_config_example_names_each_feature_out_of_scope(fdtd_lib, tmp_path):
    text = open(os.path.join(REF, "src/wavesolver/config_examples/config.xml")).read()
    expected = [("acoustic_shaders", "acoustic_shaders"), ("rigid_sound_object", "rigid_sound_object"),
                ("rigid_object_sequence", "rigid_object_sequence")]
    for element, word in expected:
        p = tmp_path / "config.xml"
        p.write_text(text)
        with pytest.raises(FDTDError) as e:
            _read(p)
        assert e.value.status == UNSUP and word in str(e.value), (element, str(e.value))
        text = _strip(text, element)
    p.write_text(text)
    with pytest.raises(FDTDError) as e:
        _read(p)
    assert e.value.status == UNSUP and "time_parallel" in str(e.value)
    text = text.replace('time_parallel="1"', 'time_parallel="0"')
    p.write_text(text)
    sc = _read(p)
    assert sc.divisions == (80, 80, 80) and sc.cell_size == 0.0005 and sc.pml_width == 0
    assert sc.boundary_handling == S.BOUNDARY_FULLY_COUPLED and len(sc.constraints) == 1
    assert sc.n_listeners == 3 and len(sc.sources) == 1 and abs(sc.sources[0].width_time - 2e-6) < 1e-20
    # PML_width="0": every side takes the Engquist-Majda update, which the solver accepts
    from acoustics_b200.batch import scene_info
    assert scene_info(sc) is not None


def ball_plane_scene(mesh, steps=3):
    """test_FDTD_RigidObject.xml in the current schema: its four balls (radius 5,
    10, 15, 10 cm from the 5 cm fixture mesh scaled) at its positions, its solver
    settings (1 m domain, h = 1 cm, PML 10, source at y = 0.4 m)."""
    h = 0.01
    sc = S.Scene(cell_size=h, divisions=(100, 100, 100), time_step=1.0 / 176400, pml_width=10, density=1.0,
                 steps=steps, name="ball_plane_scene")
    for scale, y in ((1.0, -0.4), (2.0, -0.25), (3.0, 0.0), (2.0, 0.25)):
        sc.meshes.append(S.TriangleMesh(mesh.vertices * scale, mesh.triangles))
        sc.objects.append(S.RigidObject(S.SHAPE_MESH, (0.0, y, 0.0), (0, 0, 0), mesh=len(sc.meshes) - 1))
    sc.sources.append(S.GaussianSource((0.0, 0.4, 0.0), 0.00005))
    sc.listeners = np.array([[0.2, 0.3, 0.0], [-0.2, 0.0, 0.1], [0.0, -0.1, 0.25]])
    return sc


def test_ball_plane_scene(fdtd_lib, oracle_lib, tmp_path):
    path = os.path.join(REF, "work/meshes/ball_plane_scene/test_FDTD_RigidObject.xml")
    with pytest.raises(FDTDError) as e:
        _read(path)
    assert e.value.status == INVAL and "solver_control_policy" in str(e.value)
    # the same scene in the current schema, meshes from the fixture
    mesh_dir = os.path.join(REF, "work/meshes/small_ball")
    objs = "\n".join(
        f'<rigid_object working_directory="{mesh_dir}" object_prefix="small_ball" id="{i}" fieldresolution="400" '
        f'scale="{s}" initial_position_x="0.0" initial_position_y="{y}" initial_position_z="0.0"/>'
        for i, (s, y) in enumerate(((1.0, -0.4), (2.0, -0.25), (3.0, 0.0), (2.0, 0.25))))
    p = tmp_path / "scene.xml"
    p.write_text(f"""<?xml version="1.0" ?>
<impulse_response>
  <solver sound_speed="343.0" density="1.0" cellsize="0.01" stop_time="0.01" timestepfrequency="176400"
          PML_width="10" PML_strength="1000000.0"/>
  <solver_control_policy type="static" gridresolution="100"/>
  <scene>{objs}</scene>
  <pressure_source><gaussian_pressure_source source_width_time="0.00005" source_position_x="0.0"
      source_position_y="0.4" source_position_z="0.0"/></pressure_source>
</impulse_response>
""")
    sc = _read(p)
    assert len(sc.objects) == 4 and len(sc.meshes) == 4
    assert all(o.shape == S.SHAPE_MESH for o in sc.objects)
    assert np.isclose(np.abs(sc.meshes[2].vertices).max(), 0.15)
    o = oracle_lib.OracleSolver(sc)
    o.step(2)
    flags, faces = o.classification()
    assert len(faces) > 1000 and set(np.unique(faces["boundary_object"])) == {0, 1, 2, 3}


@pytest.mark.parametrize("rel", ["work/meshes/small_ball/small_ball.obj", "work/ball/ball.obj", "work/bowl/bowl.obj"])
def test_fixture_meshes_are_closed(fdtd_lib, rel):
    import ctypes as C

    from acoustics_b200.solver import read_obj
    m = read_obj(os.path.join(REF, rel))
    md = S.MeshDesc()
    v = np.ascontiguousarray(m.vertices)
    t = np.ascontiguousarray(m.triangles)
    md.n_vertices, md.n_triangles = v.shape[0], t.shape[0]
    md.vertices = v.ctypes.data_as(C.POINTER(C.c_double))
    md.triangles = t.ctypes.data_as(C.POINTER(C.c_int32))
    centre = (v.min(axis=0) + v.max(axis=0)) / 2
    far = centre + 10 * (v.max(axis=0) - v.min(axis=0))
    pts = np.ascontiguousarray(np.vstack([centre, far]))
    out = np.zeros(2)
    assert fdtd_lib.fdtd_mesh_signed_distance(C.byref(md), 2, pts.ctypes.data, out.ctypes.data) == 0
    assert out[1] > 0  # outside is positive
    if "bowl" not in rel:
        assert out[0] < 0  # the centre of a ball is inside


def test_committed_mesh_fixture_equals_the_file(fdtd_lib):
    from acoustics_b200.solver import read_obj
    m = read_obj(os.path.join(REF, "work/meshes/small_ball/small_ball.obj"))
    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "small_ball_mesh.npz"))
    assert np.array_equal(f["vertices"], m.vertices) and np.array_equal(f["triangles"], m.triangles)
