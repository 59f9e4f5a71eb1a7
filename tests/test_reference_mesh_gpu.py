"""The reference's fixture mesh (work/meshes/small_ball/small_ball.obj,
committed as tests/golden/small_ball_mesh.npz) in the layout of its
test_FDTD_RigidObject.xml scene (four balls of 5 to 15 cm, 100^3 cells of
1 cm, PML 10) against the FP64 oracle: classification and every ghost-face
record bit-exact, pressure field within 1e-12 (FP64) and 1e-4 (FP32)."""
import os

import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.solver import PML_WaveSolver
from tests._util import rel_l2
from tests.test_reference_fixtures_cpu import ball_plane_scene

pytestmark = pytest.mark.gpu


def fixture_mesh():
    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "small_ball_mesh.npz"))
    return S.TriangleMesh(f["vertices"], f["triangles"])


@pytest.mark.parametrize("precision,tol", [(S.PRECISION_FP64, 1e-12), (S.PRECISION_FP32_COMPENSATED, 1e-4)])
def test_reference_ball_scene(oracle_lib, fdtd_lib, precision, tol):
    sc = ball_plane_scene(fixture_mesh(), steps=4)
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc, precision=precision)
    o.step(sc.steps)
    g.step(sc.steps)
    fo, go = o.classification()
    fg, gg = g.GetGrid()
    assert len(go) > 1000
    assert np.array_equal(fo, fg)
    assert np.array_equal(go, gg)
    po = o.field(S.FIELD_PRESSURE)
    assert np.abs(po).max() > 0
    assert rel_l2(g.field(S.FIELD_PRESSURE), po) <= tol
