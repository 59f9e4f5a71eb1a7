"""The configurations at their real sizes against the FP64 oracle.

* Configuration 2 (256^3, 16-cell PML, sphere + box + ellipsoid with Gaussian
  boundary acceleration, 64 listeners) for 600 steps: classification flags and
  every ghost-face record bit-exact, FP64 listener series and the pressure
  fields within 1e-12 relative L2, FP32 compensated within 1e-4.
* Two spheres on ballistic paths that touch, overlap and separate again inside
  the tested window (configuration 5's contact event on a reduced grid):
  classification bit-exact after every step, FP64 within 1e-12 through the
  contact, FP32 within 1e-4.
* Members of the batched configuration 3 at their real sizes and step counts
  (grid edges in [48, 160]) stepped as one batch: FP64 within 1e-12 of the
  oracle, FP32 within 1e-4.
"""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.batch import SolveBatch
from acoustics_b200.solver import PML_WaveSolver
from tests._util import rel_l2

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_FP32 = 1e-4


def _same_classification(o, g):
    fo, go = o.classification()
    fg, gg = g.GetGrid()
    return np.array_equal(fo, fg) and np.array_equal(go, gg), len(go)


def test_config2_full_size_against_oracle(oracle_lib, fdtd_lib):
    steps = 600
    sc = S.config2(steps=steps)
    o = oracle_lib.OracleSolver(sc)
    yo = o.step(steps)
    # the boundary pulse (t0 = 190 steps) reaches most of the 64 listeners by step 600
    assert np.count_nonzero(np.abs(yo).max(axis=0) > 1e-3 * np.abs(yo).max()) >= 32
    g64 = PML_WaveSolver(sc, precision=S.PRECISION_FP64, graph_steps=16)
    y64 = g64.step(steps)
    same, n_faces = _same_classification(o, g64)
    assert same and n_faces > 1000
    e64 = rel_l2(y64, yo)
    print(f"config 2, {steps} steps: FP64 listener rel L2 {e64:.2e}, {n_faces} ghost faces bit-exact")
    assert e64 <= TOL_FP64
    for which in (S.FIELD_PRESSURE, S.FIELD_PRESSURE_PREV):
        assert rel_l2(g64.field(which), o.field(which)) <= TOL_FP64, which
    g64.close()
    g32 = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED, graph_steps=16)
    y32 = g32.step(steps)
    same32, _ = _same_classification(o, g32)
    assert same32
    e32 = rel_l2(y32, yo)
    print(f"config 2, {steps} steps: FP32 compensated listener rel L2 {e32:.2e}")
    assert e32 <= TOL_FP32
    assert rel_l2(g32.field(S.FIELD_PRESSURE), o.field(S.FIELD_PRESSURE)) <= TOL_FP32
    g32.close()
    o.close()


def contact_scene(steps=240):
    """Two spheres (r = 1 cm) approaching along x at 60 m/s each on rows 12 mm
    apart in y: they touch when their x offset is 16 mm, overlap, and separate
    again once it is -16 mm (about steps 110 and 190 of 240)."""
    h = 0.004
    sc = S.Scene(cell_size=h, divisions=(56, 40, 40), time_step=S.reference_time_step(h), pml_width=6,
                 steps=steps, name="contact_small")
    r = 0.01
    sc.objects.append(S.RigidObject(S.SHAPE_SPHERE, (-0.03, 0.006, 0.0), (r, 0, 0), motion=S.MOTION_BALLISTIC,
                                    velocity=(60.0, 0, 0)))
    sc.objects.append(S.RigidObject(S.SHAPE_SPHERE, (0.03, -0.006, 0.002), (r, 0, 0), motion=S.MOTION_BALLISTIC,
                                    velocity=(-60.0, 0, 0), accel_kind=S.ACCEL_GAUSSIAN_TRANSLATION,
                                    accel_amplitude=1e3, accel_t0=60 * sc.time_step, accel_tau=15 * sc.time_step,
                                    accel_dir=(0, 1, 0)))
    sc.sources.append(S.GaussianSource((0.0, 0.045, 0.0), 5e-5))
    sc.listeners = np.array([[0.0, -0.04, 0.01], [0.03, 0.03, -0.02], [-0.05, 0.0, 0.03], [0.0, 0.0, -0.045]])
    return sc


def _centre_distance(sc, t):
    a, b = sc.objects
    pa = np.asarray(a.center) + np.asarray(a.velocity) * t
    pb = np.asarray(b.center) + np.asarray(b.velocity) * t
    return float(np.linalg.norm(pa - pb))


@pytest.mark.parametrize("precision,tol", [(S.PRECISION_FP64, TOL_FP64), (S.PRECISION_FP32_COMPENSATED, TOL_FP32)])
def test_spheres_touch_and_separate(oracle_lib, fdtd_lib, precision, tol):
    sc = contact_scene()
    k, r = sc.time_step, sc.objects[0].size[0]
    d = [_centre_distance(sc, (n + 1) * k) for n in range(sc.steps)]
    assert d[0] > 2 * r and min(d) < 2 * r - 0.002 and d[-1] > 2 * r  # apart, overlapping, apart
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc, precision=precision)
    yo, yg = [], []
    for n in range(sc.steps):
        yo.append(o.step(1))
        yg.append(g.step(1))
        same, _ = _same_classification(o, g)
        assert same, f"classification differs after step {n + 1}"
    yo, yg = np.concatenate(yo), np.concatenate(yg)
    assert np.abs(yo).max() > 0
    err = rel_l2(yg, yo)
    print(f"contact, {sc.steps} steps, precision {precision}: listener rel L2 {err:.2e}")
    assert err <= tol
    assert rel_l2(g.field(S.FIELD_PRESSURE), o.field(S.FIELD_PRESSURE)) <= tol
    g.close()
    o.close()


_ORACLE_SERIES = {}


def _oracle_series(oracle_lib, key, sc):
    if key not in _ORACLE_SERIES:
        o = oracle_lib.OracleSolver(sc)
        _ORACLE_SERIES[key] = o.step(sc.steps)
        o.close()
    return _ORACLE_SERIES[key]


@pytest.mark.parametrize("precision,tol", [(S.PRECISION_FP64, TOL_FP64), (S.PRECISION_FP32_COMPENSATED, TOL_FP32)])
def test_config3_members_full_size(oracle_lib, fdtd_lib, precision, tol):
    scenes = S.config3()
    members = (1, 3, 5, 6)                      # 0.25-0.5 M cells, 1562-2917 steps, 1-3 bodies
    pick = [scenes[i] for i in members]
    for sc in pick:
        assert all(48 <= n <= 160 for n in sc.divisions)
    with SolveBatch(pick, precision=precision, graph_steps=16) as b:
        b.run()
        ys = [b.output(m) for m in range(len(pick))]
    for m, sc in enumerate(pick):
        yo = _oracle_series(oracle_lib, ("config3", members[m]), sc)
        assert np.abs(yo).max() > 0
        err = rel_l2(ys[m], yo)
        print(f"config 3 member {m} {sc.divisions} x {sc.steps} steps: listener rel L2 {err:.2e}")
        assert err <= tol, m
