"""C-ABI of libfdtd_b200.so without a GPU: the library loads and exports every
symbol include/fdtd_c.h declares, the ctypes mirrors match the C struct
layouts, the XML scene reader and the all_audio.dat writer work, and solver
creation fails cleanly when no device is visible."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from acoustics_b200 import scene as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fdtd_c.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fdtd_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(fdtd_lib):
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(fdtd_lib, n), n
    from acoustics_b200 import _lib
    assert sorted(_lib.EXPORTS) == names


def test_abi_version(fdtd_lib):
    assert fdtd_lib.fdtd_abi_version() == 5


def test_struct_layouts_match_header(tmp_path):
    prog = tmp_path / "sizes.c"
    prog.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "fdtd_c.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(fdtd_object_desc), sizeof(fdtd_plane_desc),
         sizeof(fdtd_gaussian_source_desc), sizeof(fdtd_scene_desc), sizeof(fdtd_options),
         sizeof(fdtd_solver_info), sizeof(fdtd_ghost_face), sizeof(fdtd_server_config),
         sizeof(fdtd_server_stats));
  printf("%zu %zu %zu %zu\\n", offsetof(fdtd_scene_desc, objects), offsetof(fdtd_scene_desc, listeners),
         offsetof(fdtd_object_desc, gravity), offsetof(fdtd_solver_info, algorithmic_bytes_per_step));
  return 0;
}
""")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in out[0].split()]
    offs = [int(x) for x in out[1].split()]
    assert sizes == [C.sizeof(S.ObjectDesc), C.sizeof(S.PlaneDesc), C.sizeof(S.GaussianSourceDesc),
                     C.sizeof(S.SceneDesc), C.sizeof(S.Options), C.sizeof(S.SolverInfo), C.sizeof(S.GhostFace),
                     C.sizeof(S.ServerConfig), C.sizeof(S.ServerStats)]
    assert offs == [S.SceneDesc.objects.offset, S.SceneDesc.listeners.offset, S.ObjectDesc.gravity.offset,
                    S.SolverInfo.algorithmic_bytes_per_step.offset]
    assert S.GHOST_FACE_DTYPE.itemsize == C.sizeof(S.GhostFace)


def test_cell_dtype_matches_header(tmp_path):
    """fdtd_cell (FetchCell / SampleAxisAlignedSlice) against CELL_DTYPE, field by field."""
    fields = list(S.CELL_DTYPE.names)
    prog = tmp_path / "cell.c"
    prog.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"fdtd_c.h\"\nint main(void) {\n"
                    + '  printf("%zu\\n", sizeof(fdtd_cell));\n'
                    + "".join(f'  printf("%zu\\n", offsetof(fdtd_cell, {f}));\n' for f in fields)
                    + "  return 0;\n}\n")
    exe = tmp_path / "cell"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == S.CELL_DTYPE.itemsize
    assert out[1:] == [S.CELL_DTYPE.fields[f][1] for f in fields]


def test_gaussian_source_defaults(fdtd_lib):
    g = S.GaussianSourceDesc()
    g.width_time = 2e-4
    assert fdtd_lib.fdtd_gaussian_source_defaults(C.byref(g), C.c_double(343.0)) == 0
    assert g.width_space == pytest.approx(343.0 * 2e-4, rel=0, abs=0)
    assert g.normalize_constant == 1.0 / (np.sqrt(2.0 * np.pi) * g.width_space) ** 3


SCENE_XML = """<?xml version="1.0" ?>
<!-- minimal scene -->
<impulse_response>
  <solver sound_speed="343" density="1.184" cellsize="0.005" stop_time="0.01" number_of_timesteps="120"
          timestepfrequency="237635.4" output_pattern="out/%s" write_pressure_field_to_disk="0"
          PML_width="10" PML_strength="1000000.0"/>
  <solver_control_policy type="static" gridresolution="64" gridresolution_z="48" domain_center_x="0.01"/>
  <scene>
    <analytic_sphere center_x="0.0" center_y="0.0" center_z="0.0" radius="0.04"
                     acceleration="translation" accel_amplitude="1000" accel_t0="4e-4" accel_tau="1e-4"
                     accel_dir_x="0" accel_dir_y="0" accel_dir_z="1"/>
    <analytic_box center_x="0.05" center_y="0.0" center_z="0.0" half_x="0.02" half_y="0.01" half_z="0.005"
                  velocity_x="1.5"/>
    <constraint direction="1" sign="1" height="-0.1"/>
  </scene>
  <pressure_source>
    <gaussian_pressure_source source_width_time="2e-4" source_position_x="0.02" source_position_y="0.03"
                              source_position_z="-0.01" source_sign_flip="1"/>
  </pressure_source>
  <listening_point_list>
    <listening_point x="0.01" y="0.02" z="0.03"/>
    <listening_point x="-0.01" y="0.0" z="0.0"/>
  </listening_point_list>
</impulse_response>
"""


def test_xml_scene_reader(fdtd_lib, tmp_path):
    from acoustics_b200.solver import scene_from_xml
    p = tmp_path / "scene.xml"
    p.write_text(SCENE_XML)
    sc = scene_from_xml(str(p))
    assert tuple(sc.divisions) == (64, 64, 48)
    assert sc.cell_size == 0.005 and sc.density == 1.184 and sc.pml_width == 10
    assert sc.time_step == 1.0 / 237635.4
    assert sc.domain_center[0] == 0.01 and sc.steps == 120 and sc.end_time == 0.01
    assert len(sc.objects) == 2 and sc.objects[0].shape == S.SHAPE_SPHERE
    assert sc.objects[0].accel_kind == S.ACCEL_GAUSSIAN_TRANSLATION and sc.objects[0].accel_tau == 1e-4
    assert sc.objects[1].shape == S.SHAPE_BOX and sc.objects[1].motion == S.MOTION_BALLISTIC
    assert tuple(sc.objects[1].size) == (0.02, 0.01, 0.005)
    assert len(sc.constraints) == 1 and sc.constraints[0].height == -0.1
    src = sc.sources[0]
    assert src.width_space == 343.0 * 2e-4                      # parser default c * sigma_t
    assert src.normalize_constant == -1.0 / (np.sqrt(2.0 * np.pi) * src.width_space) ** 3  # sign flip
    assert np.array_equal(sc.listeners, [[0.01, 0.02, 0.03], [-0.01, 0.0, 0.0]])
    assert sc.boundary_handling == S.BOUNDARY_RASTERIZE
    # ImpulseResponseParser.cpp:547-555
    p.write_text(SCENE_XML.replace('<solver ', '<solver boundary_handling="fully_coupled" ', 1))
    assert scene_from_xml(str(p)).boundary_handling == S.BOUNDARY_FULLY_COUPLED


@pytest.mark.parametrize("bad,status", [
    ("<impulse_response><solver cellsize='0.005'/></impulse_response>", -1),
    ("<impulse_response>", -1),
    ("<other/>", -1),
    # a mesh object without its working_directory / object_prefix
    (SCENE_XML.replace("analytic_sphere", "rigid_sound_object", 1).replace(
        "radius=\"0.04\"", "", 1), -1),
    (SCENE_XML.replace("analytic_sphere", "rigid_object_sequence", 1).replace(
        "radius=\"0.04\"", "", 1), -7),
    (SCENE_XML.replace('type="static"', 'type="dynamic"'), -7),
    (SCENE_XML.replace('<solver ', '<solver boundary_handling="voxelized" ', 1), -1),
])
def test_xml_errors(fdtd_lib, tmp_path, bad, status):
    p = tmp_path / "bad.xml"
    p.write_text(bad)
    h = C.c_void_p()
    st = fdtd_lib.fdtd_scene_from_xml(str(p).encode(), C.byref(h))
    assert st == status
    assert fdtd_lib.fdtd_last_error()


def test_audio_writer_appends_raw_doubles(fdtd_lib, tmp_path):
    from acoustics_b200.solver import write_audio
    path = str(tmp_path / "all_audio.dat")
    a = np.arange(12, dtype=np.float64).reshape(4, 3)
    write_audio(path, a[:2])
    write_audio(path, a[2:])
    assert np.array_equal(np.fromfile(path, dtype=np.float64).reshape(4, 3), a)


def test_create_without_device_fails_cleanly(fdtd_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from acoustics_b200._lib import FDTDError
    from acoustics_b200.solver import PML_WaveSolver
    with pytest.raises(FDTDError) as e:
        PML_WaveSolver(S.config1())
    assert e.value.status == -3


def test_invalid_scenes_are_rejected_before_device_use(fdtd_lib):
    bad = []
    sc = S.config1(); sc.pml_width = -1.0; bad.append((sc, -1))
    sc = S.config1(); sc.boundary_condition_preset = 3; bad.append((sc, -1))
    sc = S.config1(); sc.air_viscosity_alpha = -0.1; bad.append((sc, -1))
    sc = S.config1(); sc.boundary_handling = 7; bad.append((sc, -1))
    sc = S.config1(); sc.boundary_handling = S.BOUNDARY_FULLY_COUPLED
    sc.objects.append(S.RigidObject(S.SHAPE_ELLIPSOID, (0.05, 0, 0), (0.01, 0.01, 0.01))); bad.append((sc, -7))
    sc = S.config1(); sc.cell_size = -1.0; bad.append((sc, -1))
    sc = S.config1(); sc.objects = [S.RigidObject(S.SHAPE_SPHERE, (0, 0, 0), (0.01, 0, 0))] * 9; bad.append((sc, -1))
    for sc, status in bad:
        desc, keep = sc.to_c()
        h = C.c_void_p()
        assert fdtd_lib.fdtd_solver_create(C.byref(desc), None, C.byref(h)) == status
        assert h.value is None


def test_server_and_batch_without_device_fail_cleanly(fdtd_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from acoustics_b200._lib import FDTDError
    from acoustics_b200.batch import SolveBatch
    from acoustics_b200.server import SolveServer
    with pytest.raises(FDTDError):
        SolveServer()
    with pytest.raises(FDTDError):
        SolveBatch()


def test_scene_device_bytes_follows_the_arena_layout(fdtd_lib):
    from acoustics_b200.batch import scene_device_bytes
    small = S.config1(divisions=(40, 36, 32), pml_width=6, radius=0.02)
    big = S.config1()
    a32, a64 = scene_device_bytes(small), scene_device_bytes(small, precision=S.PRECISION_FP64)
    assert 0 < a32 < a64 < scene_device_bytes(big, precision=S.PRECISION_FP64)
    # padded layout: rows of Nz+1 rounded up to 8, Ny+1 rows, Nx+1 planes
    npad = 41 * 37 * 40
    # per padded cell: flags 2 B, p[2] + dinc + pd[3] + 2 x 3 faces = 12 words (FP32),
    # plus the compact PML storage of the z-slab box and the small tables
    assert 12 * 4 * npad < a32 < 16 * 4 * npad + (1 << 20)
    bad = S.config1(); bad.cell_size = -1.0
    with pytest.raises(Exception):
        scene_device_bytes(bad)


def test_scene_info_on_the_host(fdtd_lib):
    from acoustics_b200.batch import scene_info
    sc = S.config2(n=256)
    i32, i64 = scene_info(sc), scene_info(sc, precision=S.PRECISION_FP64)
    assert tuple(i32.divisions) == (256, 256, 256)
    assert i32.n_interior_cells == 11239424 and i32.n_pml_cells == 5537792
    assert i32.algorithmic_bytes_per_step == 444989440.0
    assert i64.algorithmic_bytes_per_step == 2 * i32.algorithmic_bytes_per_step


def test_matrix_file_layout(fdtd_lib, tmp_path):
    """IO::writeMatrixX BINARY / MATRIX::write layout: int32 rows, int32 cols,
    row-major doubles; the reader returns the same array."""
    from acoustics_b200.solver import read_matrix, write_matrix
    a = np.arange(12, dtype=np.float64).reshape(4, 3) * 0.5 - 1.0
    p = str(tmp_path / "m.dat")
    write_matrix(p, a)
    raw = open(p, "rb").read()
    assert np.frombuffer(raw[:8], dtype=np.int32).tolist() == [4, 3]
    assert np.array_equal(np.frombuffer(raw[8:], dtype=np.float64), a.ravel())
    assert len(raw) == 8 + 12 * 8
    assert np.array_equal(read_matrix(p), a)
    with pytest.raises(Exception):
        read_matrix(str(tmp_path / "missing.dat"))
