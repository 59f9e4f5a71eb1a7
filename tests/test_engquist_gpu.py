"""Sides without PML: boundary presets 1 (walls +x, +z) and 2 (PML on +z only),
and a PML under 1.5 cells, where the reference's Engquist-Majda update of the
cells one cell inside the domain edge is live (MAC_Grid.cpp:515-920,
:4027-4101).  The CUDA path against the FP64 oracle: listener series and the
current and previous pressure fields (the exterior cells carry the values the
reference's three rotating buffers hold) within 1e-12 in FP64, 1e-4 in FP32;
graphs, snapshot / restore, a moving body; a solid inside an Engquist stencil
is reported, not computed."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200._lib import FDTDError
from acoustics_b200.solver import PML_WaveSolver
from tests._util import rel_l2

pytestmark = pytest.mark.gpu

F64, F32 = S.PRECISION_FP64, S.PRECISION_FP32_COMPENSATED
TOL = {F64: 1e-12, F32: 1e-4}


def wall_scene(preset, pml=5.0, n=(36, 32, 40), steps=300, near_wall_listener=True):
    """A sphere, a source and listeners (two of them within two cells of a side
    without PML, so their MLS stencils reach the exterior cells)."""
    h = 0.005
    sc = S.Scene(cell_size=h, divisions=n, time_step=S.reference_time_step(h), pml_width=pml, steps=steps,
                 name=f"walls_preset{preset}")
    sc.boundary_condition_preset = preset
    sc.objects.append(S.RigidObject(S.SHAPE_SPHERE, (0.005, -0.004, 0.003), (0.015, 0, 0)))
    sc.sources.append(S.GaussianSource((0.04, 0.02, 0.045), 1e-4))
    half = np.asarray(n) * h / 2
    lis = [[-0.03, 0.03, -0.02], [0.02, -0.02, 0.03], [0.0, 0.035, 0.0]]
    if near_wall_listener:
        lis.append([half[0] - 1.3 * h, 0.01, 0.0])     # +x side
        lis.append([0.01, -0.01, half[2] - 1.6 * h])   # +z side
    sc.listeners = np.array(lis)
    return sc


def _compare(oracle_lib, sc, precision, steps, **kw):
    o = oracle_lib.OracleSolver(sc)
    yo = o.step(steps)
    g = PML_WaveSolver(sc, precision=precision, **kw)
    yg = g.step(steps)
    assert np.abs(yo).max() > 0
    assert rel_l2(yg, yo) <= TOL[precision], rel_l2(yg, yo)
    for f in (S.FIELD_PRESSURE, S.FIELD_PRESSURE_PREV):
        if precision == F32 and f == S.FIELD_PRESSURE_PREV:
            continue
        a, b = g.field(f), o.field(f)
        assert rel_l2(a, b) <= TOL[precision], (f, rel_l2(a, b))
    return g, o


@pytest.mark.parametrize("preset", [1, 2])
@pytest.mark.parametrize("precision", [F64, F32])
def test_wall_presets_against_oracle(oracle_lib, fdtd_lib, preset, precision):
    sc = wall_scene(preset)
    g, _ = _compare(oracle_lib, sc, precision, sc.steps)
    g.close()


@pytest.mark.parametrize("pml", [1.0, 0.0])
def test_thin_pml_reaches_engquist(oracle_lib, fdtd_lib, pml):
    """Preset 0 with a PML under 1.5 cells: the cells one inside the edge are
    not PML cells (pml 1: their exterior cells are; pml 0: no cell is)."""
    sc = wall_scene(0, pml=pml, steps=200)
    _compare(oracle_lib, sc, F64, sc.steps)


def test_walls_with_graphs(oracle_lib, fdtd_lib):
    sc = wall_scene(1, steps=256)
    _compare(oracle_lib, sc, F64, sc.steps, graph_steps=16)


def test_walls_snapshot_restore(fdtd_lib):
    """The history of exterior values travels with the snapshot."""
    sc = wall_scene(2, steps=200)
    a = PML_WaveSolver(sc)
    ya = a.step(200)
    b = PML_WaveSolver(sc)
    y1 = b.step(80)
    blob = b.snapshot()
    c = PML_WaveSolver(sc)
    c.restore(blob)
    y2 = c.step(120)
    assert np.array_equal(ya, np.concatenate([y1, y2]))
    assert np.array_equal(a.field(S.FIELD_PRESSURE), c.field(S.FIELD_PRESSURE))


def test_walls_moving_body(oracle_lib, fdtd_lib):
    sc = wall_scene(2, steps=160)
    sc.objects[0] = S.RigidObject(S.SHAPE_SPHERE, (-0.01, 0.0, 0.0), (0.012, 0, 0), motion=S.MOTION_BALLISTIC,
                                  velocity=(25.0, 10.0, 0.0))
    _compare(oracle_lib, sc, F64, sc.steps)
    _compare(oracle_lib, sc, F32, sc.steps)


def test_solid_in_engquist_stencil_is_reported(fdtd_lib):
    sc = wall_scene(1, steps=5, near_wall_listener=False)
    half = np.asarray(sc.divisions) * sc.cell_size / 2
    # a sphere touching the +x side's Engquist cells
    sc.objects.append(S.RigidObject(S.SHAPE_SPHERE, (half[0] - 0.012, 0.0, -0.03), (0.0105, 0, 0)))
    g = PML_WaveSolver(sc)
    with pytest.raises(FDTDError) as e:
        g.step(2)
    assert e.value.status == S.STATUS_CODE["FDTD_ERR_UNSUPPORTED"]
    assert "Engquist" in str(e.value)


def test_walls_not_batched(fdtd_lib):
    from acoustics_b200.batch import SolveBatch
    b = SolveBatch(precision=F32)
    with pytest.raises(FDTDError) as e:
        b.add(wall_scene(1, steps=10), 10)
    assert "PML on every side" in str(e.value)
    b.close()
