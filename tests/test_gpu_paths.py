"""GPU paths against the FP64 oracle through the C-ABI: FP32 compensated,
plain (phased) FP64, CUDA graphs, snapshot/restore, accelerating bodies,
plane constraints and moving bodies."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.solver import PML_WaveSolver
from tests._util import rel_l2, small_config2

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_FP32 = 1e-4


def test_fp32_compensated_config1(oracle_lib, fdtd_lib):
    sc = S.config1()
    yo = oracle_lib.OracleSolver(sc).step(500)
    g = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED)
    yg = g.step(500)
    err = rel_l2(yg, yo)
    print("cfg1 fp32 listener rel L2", err)
    assert err <= TOL_FP32


def test_phased_fp64_matches_oracle(oracle_lib, fdtd_lib):
    sc = S.config1()
    yo = oracle_lib.OracleSolver(sc).step(200)
    g = PML_WaveSolver(sc, kernel=S.KERNEL_PHASED)
    yg = g.step(200)
    assert rel_l2(yg, yo) <= TOL_FP64


@pytest.mark.parametrize("precision", [S.PRECISION_FP64, S.PRECISION_FP32_COMPENSATED])
def test_graph_replay_identical_to_eager(fdtd_lib, precision):
    sc = S.config1(divisions=(48, 40, 56), pml_width=8, radius=0.025)
    a = PML_WaveSolver(sc, precision=precision).step(75)
    b = PML_WaveSolver(sc, precision=precision, graph_steps=10).step(75)
    assert np.array_equal(a, b)
    # graphs captured ahead of time by prepare_graphs replay the same steps
    c = PML_WaveSolver(sc, precision=precision, graph_steps=10)
    y0 = c.step(5)
    c.prepare_graphs()
    assert np.array_equal(np.concatenate([y0, c.step(70)]), a)


def test_snapshot_restore_roundtrip(fdtd_lib):
    sc = S.config1()
    g = PML_WaveSolver(sc)
    g.step(40)
    blob = g.snapshot()
    y1 = g.step(30)
    g.restore(blob)
    y2 = g.step(30)
    assert np.array_equal(y1, y2)


def test_accelerating_bodies_fp64(oracle_lib, fdtd_lib):
    sc = small_config2()
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc)
    yo, yg = o.step(sc.steps), g.step(sc.steps)
    assert np.abs(yo).max() > 0
    assert rel_l2(yg, yo) <= TOL_FP64
    fo, go = o.classification()
    fg, gg = g.GetGrid()
    assert np.array_equal(fo, fg)
    assert np.array_equal(go, gg)


def test_accelerating_bodies_fp32(oracle_lib, fdtd_lib):
    sc = small_config2()
    yo = oracle_lib.OracleSolver(sc).step(sc.steps)
    yg = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED).step(sc.steps)
    assert rel_l2(yg, yo) <= TOL_FP32


def test_plane_constraint_and_pml_overlap(oracle_lib, fdtd_lib):
    sc = S.config1(divisions=(40, 40, 40), pml_width=6, radius=0.02)
    sc.constraints.append(S.PlaneConstraint(1, 1, -0.05))       # floor at y = -5 cm
    sc.objects.append(S.RigidObject(S.SHAPE_BOX, (0.07, 0.0, 0.0), (0.04, 0.02, 0.02)))  # reaches into the PML
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc)
    yo, yg = o.step(120), g.step(120)
    fo, go = o.classification()
    fg, gg = g.GetGrid()
    assert np.array_equal(fo, fg)
    assert np.array_equal(go, gg)
    assert rel_l2(yg, yo) <= TOL_FP64
    assert rel_l2(g.field(S.FIELD_PRESSURE), o.field(S.FIELD_PRESSURE)) <= TOL_FP64


def moving_scene(steps=160):
    sc = S.Scene(cell_size=0.004, divisions=(48, 40, 40), time_step=S.reference_time_step(0.004), pml_width=6,
                 steps=steps, name="moving_small")
    k = sc.time_step
    # two spheres approaching at ~30 m/s (0.013 cells per step)
    sc.objects.append(S.RigidObject(S.SHAPE_SPHERE, (-0.03, 0.0, 0.0), (0.012, 0, 0), motion=S.MOTION_BALLISTIC,
                                    velocity=(60.0, 0, 0), gravity=(0, 0, -9.81)))
    sc.objects.append(S.RigidObject(S.SHAPE_BOX, (0.035, 0.005, 0.0), (0.01, 0.008, 0.008), motion=S.MOTION_BALLISTIC,
                                    velocity=(-60.0, 0, 0), accel_kind=S.ACCEL_GAUSSIAN_TRANSLATION,
                                    accel_amplitude=1e3, accel_t0=40 * k, accel_tau=10 * k, accel_dir=(1, 0, 0)))
    sc.sources.append(S.GaussianSource((0.0, 0.04, 0.0), 5e-5))
    sc.listeners = np.array([[0.0, -0.03, 0.01], [0.02, 0.02, -0.02], [-0.04, 0.0, 0.03]])
    return sc


@pytest.mark.parametrize("precision,tol", [(S.PRECISION_FP64, TOL_FP64), (S.PRECISION_FP32_COMPENSATED, TOL_FP32)])
def test_moving_bodies(oracle_lib, fdtd_lib, precision, tol):
    sc = moving_scene()
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc, precision=precision)
    for chunk in range(4):
        yo, yg = o.step(40), g.step(40)
        assert rel_l2(yg, yo) <= tol, chunk
        fo, go = o.classification()
        fg, gg = g.GetGrid()
        assert np.array_equal(fo, fg), chunk
        assert np.array_equal(go, gg), chunk


def test_moving_bodies_reduced_pml_state(oracle_lib, fdtd_lib):
    """Moving bodies that stay clear of the PML until end_time keep the reduced
    PML state: classification bit-exact after every chunk,
    listener series within 1e-4 of the FP64 oracle and 1e-5 of the full state."""
    sc = moving_scene()
    sc.end_time = sc.steps * sc.time_step
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED)
    f = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED, pml_state=S.PML_STATE_FULL)
    assert g.pml_state() == S.PML_STATE_AUTO and f.pml_state() == S.PML_STATE_FULL
    assert g.shell_staging() == S.SHELL_STAGING_RING  # beside the classification: the per-thread kernel
    yo, yg, yf = [], [], []
    for chunk in range(4):
        yo.append(o.step(40))
        yg.append(g.step(40))
        yf.append(f.step(40))
        fo, go = o.classification()
        fg, gg = g.GetGrid()
        assert np.array_equal(fo, fg), chunk
        assert np.array_equal(go, gg), chunk
    yo, yg, yf = np.concatenate(yo), np.concatenate(yg), np.concatenate(yf)
    assert rel_l2(yg, yo) <= TOL_FP32
    assert rel_l2(yg, yf) <= 1e-5
    assert g.overlapped_steps() > 0


def test_reduced_pml_state_fp32(oracle_lib, fdtd_lib):
    """FP32 static solves keep the reduced PML state (one leapfrog increment for
    the axes without absorption of a PML cell): listener series and pressure
    field agree with the FP64 oracle and with the full split state."""
    from acoustics_b200._lib import FDTDError
    sc = small_config2()
    o = oracle_lib.OracleSolver(sc)
    yo = o.step(sc.steps)
    red = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED)
    full = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED, pml_state=S.PML_STATE_FULL)
    assert red.pml_state() == S.PML_STATE_AUTO
    assert full.pml_state() == S.PML_STATE_FULL
    yr, yf = red.step(sc.steps), full.step(sc.steps)
    print("reduced vs oracle", rel_l2(yr, yo), "full vs oracle", rel_l2(yf, yo), "reduced vs full", rel_l2(yr, yf))
    assert rel_l2(yr, yo) <= TOL_FP32
    assert rel_l2(yf, yo) <= TOL_FP32
    assert rel_l2(yr, yf) <= 1e-5
    assert rel_l2(red.field(S.FIELD_PRESSURE), o.field(S.FIELD_PRESSURE)) <= TOL_FP32
    with pytest.raises(FDTDError):
        red.field(S.FIELD_PML_PX)


def test_reduced_pml_state_only_where_exact(fdtd_lib):
    """The full state stays where the reduction would not be exact: FP64,
    moving bodies, a solid cell inside the PML, and a PML width whose inner
    faces carry absorption next to non-PML cells."""
    f32 = S.PRECISION_FP32_COMPENSATED
    assert PML_WaveSolver(S.config1(), precision=f32).pml_state() == S.PML_STATE_AUTO
    assert PML_WaveSolver(S.config1()).pml_state() == S.PML_STATE_FULL
    assert PML_WaveSolver(moving_scene(), precision=f32).pml_state() == S.PML_STATE_FULL
    sc = S.config1(divisions=(40, 40, 40), pml_width=6, radius=0.02)
    sc.objects.append(S.RigidObject(S.SHAPE_BOX, (0.07, 0.0, 0.0), (0.04, 0.02, 0.02)))  # reaches into the PML
    assert PML_WaveSolver(sc, precision=f32).pml_state() == S.PML_STATE_FULL
    assert PML_WaveSolver(S.config1(pml_width=6.5), precision=f32).pml_state() == S.PML_STATE_AUTO
    assert PML_WaveSolver(S.config1(pml_width=6.2), precision=f32).pml_state() == S.PML_STATE_FULL


@pytest.mark.parametrize("pml_width", [6.5, 6.2])
def test_fp32_fractional_pml_width(oracle_lib, fdtd_lib, pml_width):
    sc = S.config1(divisions=(40, 36, 44), pml_width=pml_width, radius=0.02)
    yo = oracle_lib.OracleSolver(sc).step(150)
    yg = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED).step(150)
    assert rel_l2(yg, yo) <= TOL_FP32


@pytest.mark.parametrize("kernel,precision,tol", [(S.KERNEL_FUSED, S.PRECISION_FP64, TOL_FP64),
                                                  (S.KERNEL_PHASED, S.PRECISION_FP64, TOL_FP64),
                                                  (S.KERNEL_FUSED, S.PRECISION_FP32_COMPENSATED, TOL_FP32)])
def test_air_viscosity(oracle_lib, fdtd_lib, kernel, precision, tol):
    """alpha > 0: the update of a cell with a valid history adds
    c alpha k (lap^n - lap^{n-1}) (MAC_Grid.cpp:926-930)."""
    sc = S.config1(divisions=(40, 36, 44), pml_width=6, radius=0.02)
    sc.air_viscosity_alpha = 2e-5
    yo = oracle_lib.OracleSolver(sc).step(200)
    yg = PML_WaveSolver(sc, precision=precision, kernel=kernel).step(200)
    assert rel_l2(yg, yo) <= tol
    sc.air_viscosity_alpha = 0.0
    y0 = oracle_lib.OracleSolver(sc).step(200)
    assert rel_l2(yo, y0) > 1e-4  # the term is visible


def test_air_viscosity_moving_bodies(oracle_lib, fdtd_lib):
    sc = moving_scene(steps=80)
    sc.air_viscosity_alpha = 2e-5
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc)
    yo, yg = o.step(80), g.step(80)
    assert rel_l2(yg, yo) <= TOL_FP64


@pytest.mark.parametrize("precision,tol", [(S.PRECISION_FP64, TOL_FP64), (S.PRECISION_FP32_COMPENSATED, TOL_FP32)])
def test_config5_full_size_first_steps(oracle_lib, fdtd_lib, precision, tol):
    """Configuration 5 at full size (384x384x256, two ballistic spheres, per-step
    reclassification): the first steps against the FP64 oracle, classification
    bit-exact after every step."""
    sc = S.config5(steps=6)
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc, precision=precision)
    ys_o, ys_g = [], []
    for step in range(6):
        ys_o.append(o.step(1))
        ys_g.append(g.step(1))
        fo, go = o.classification()
        fg, gg = g.GetGrid()
        assert np.array_equal(fo, fg), step
        assert np.array_equal(go, gg), step
    assert rel_l2(np.concatenate(ys_g), np.concatenate(ys_o)) <= tol
    # the pulse has not reached the listeners yet: compare the whole pressure field
    assert rel_l2(g.field(S.FIELD_PRESSURE), o.field(S.FIELD_PRESSURE)) <= tol
    # the spheres stay clear of the PML: every step ran its shell beside the classification
    assert g.overlapped_steps() == 6


@pytest.mark.parametrize("precision", [S.PRECISION_FP64, S.PRECISION_FP32_COMPENSATED])
def test_long_host_call_staging(fdtd_lib, precision):
    """One host call of 700 steps with 16-step graphs (more rows than the pinned
    staging buffer holds, the classifying step first) gives the rows that the
    device-output call writes, bit for bit."""
    import torch
    sc = S.config1()
    n = 700
    a = PML_WaveSolver(sc, precision=precision, graph_steps=16)
    ya = a.step(n)
    b = PML_WaveSolver(sc, precision=precision, graph_steps=16)
    buf = torch.zeros((n, sc.listeners.shape[0]), dtype=torch.float64, device="cuda")
    b.step_device(n, buf.data_ptr())
    b.synchronize()
    assert np.abs(ya).max() > 0
    assert np.array_equal(ya, buf.cpu().numpy())
    a.close()
    b.close()


def test_kept_device_blocks_start_clean(fdtd_lib):
    """A destroyed solver's device block serves the next solver, which starts
    from the same zero state: rows equal those of the first run; the kept
    blocks can be released."""
    sc = S.config1()
    a = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED)
    ya = a.step(120)
    a.close()
    b = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED)
    yb = b.step(120)
    b.close()
    assert np.abs(ya).max() > 0 and np.array_equal(ya, yb)
    fdtd_lib.fdtd_release_cached_memory(-1)
    c = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED)
    assert np.array_equal(c.step(120), ya)
    c.close()
