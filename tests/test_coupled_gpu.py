"""FULLY_COUPLED ghost cells (MAC_Grid::PML_pressureUpdateGhostCells with
boundary_handling="fully_coupled"): image-point interpolation of every ghost
face and the coupled sparse solve, on the GPU against the FP64 oracle's
restatement of the same algorithm."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200._lib import FDTDError
from acoustics_b200.solver import PML_WaveSolver
from tests._util import rel_l2

pytestmark = pytest.mark.gpu

TOL_FC64 = 1e-11  # the coupled solves stop at one machine epsilon; weights come from different factorizations
TOL_FP32 = 1e-4


def fc_scene():
    sc = S.config1(divisions=(40, 36, 44), pml_width=6, radius=0.03)
    sc.objects.append(S.RigidObject(S.SHAPE_BOX, (0.05, -0.04, 0.02), (0.02, 0.015, 0.01),
                                    accel_kind=S.ACCEL_GAUSSIAN_TRANSLATION, accel_amplitude=1e3,
                                    accel_t0=3e-4, accel_tau=8e-5, accel_dir=(0.6, 0.8, 0.0)))
    sc.boundary_handling = S.BOUNDARY_FULLY_COUPLED
    return sc


@pytest.mark.parametrize("precision,tol", [(S.PRECISION_FP64, TOL_FC64), (S.PRECISION_FP32_COMPENSATED, TOL_FP32)])
def test_fully_coupled_matches_oracle(oracle_lib, fdtd_lib, precision, tol):
    sc = fc_scene()
    yo = oracle_lib.OracleSolver(sc).step(200)
    g = PML_WaveSolver(sc, precision=precision)
    yg = g.step(200)
    info = g.boundary_info()
    print(precision, "rel L2", rel_l2(yg, yo), info)
    assert info["immersed"] > 0 and info["iterations"] > 0
    assert rel_l2(yg, yo) <= tol


def test_fully_coupled_differs_from_rasterize(fdtd_lib):
    sc = fc_scene()
    yc = PML_WaveSolver(sc).step(150)
    sc.boundary_handling = S.BOUNDARY_RASTERIZE
    yr = PML_WaveSolver(sc).step(150)
    d = rel_l2(yc, yr)
    assert 1e-5 < d < 0.1, d


def test_fully_coupled_only_where_built(fdtd_lib):
    sc = fc_scene()
    with pytest.raises(FDTDError):
        PML_WaveSolver(sc, kernel=S.KERNEL_PHASED)
    sc.objects.append(S.RigidObject(S.SHAPE_ELLIPSOID, (0.0, 0.05, 0.0), (0.01, 0.008, 0.006)))
    with pytest.raises(FDTDError):  # no closest-point query for ellipsoids
        PML_WaveSolver(sc)


@pytest.mark.parametrize("precision,tol", [(S.PRECISION_FP64, TOL_FC64), (S.PRECISION_FP32_COMPENSATED, TOL_FP32)])
def test_fully_coupled_mesh_bodies(oracle_lib, fdtd_lib, precision, tol):
    """Mesh bodies: an icosphere and a box mesh, reflected through their hierarchies."""
    sc = fc_scene()
    sc.objects = []
    sc.meshes = [S.icosphere(0.025, level=2), S.box_mesh((0.02, 0.015, 0.01))]
    sc.objects.append(S.RigidObject(S.SHAPE_MESH, (0.0, 0.0, 0.0), (0, 0, 0), mesh=0))
    sc.objects.append(S.RigidObject(S.SHAPE_MESH, (0.05, -0.04, 0.02), (0, 0, 0), mesh=1,
                                    accel_kind=S.ACCEL_GAUSSIAN_TRANSLATION, accel_amplitude=1e3,
                                    accel_t0=3e-4, accel_tau=8e-5, accel_dir=(0.6, 0.8, 0.0)))
    yo = oracle_lib.OracleSolver(sc).step(150)
    g = PML_WaveSolver(sc, precision=precision)
    yg = g.step(150)
    assert g.boundary_info()["immersed"] > 0
    assert rel_l2(yg, yo) <= tol


@pytest.mark.parametrize("precision,tol", [(S.PRECISION_FP64, TOL_FC64), (S.PRECISION_FP32_COMPENSATED, TOL_FP32)])
def test_fully_coupled_moving_bodies(oracle_lib, fdtd_lib, precision, tol):
    """A moving sphere beside the static box: the coupled rows are rebuilt every step."""
    sc = fc_scene()
    sc.objects[0] = S.RigidObject(S.SHAPE_SPHERE, (-0.02, 0.0, 0.0), (0.025, 0, 0), motion=S.MOTION_BALLISTIC,
                                  velocity=(40.0, 0, 0))
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc, precision=precision)
    for chunk in range(3):
        yo, yg = o.step(30), g.step(30)
        fo, go = o.classification()
        fg, gg = g.GetGrid()
        assert np.array_equal(fo, fg) and np.array_equal(go, gg), chunk
        assert rel_l2(yg, yo) <= tol, chunk
    assert g.boundary_info()["immersed"] > 0
