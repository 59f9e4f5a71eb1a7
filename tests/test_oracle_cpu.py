"""The FP64 CPU oracle against known answers, an independent numpy restatement
and the committed golden fixtures (CPU only)."""
import math
import os

import numpy as np
import pytest

from acoustics_b200 import scene as S
from tests._util import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))


def small_scene(n=(24, 20, 28), steps=40, with_sphere=True):
    h = 0.005
    sc = S.Scene(cell_size=h, divisions=n, time_step=S.reference_time_step(h), pml_width=4, steps=steps,
                 name="small")
    if with_sphere:
        sc.objects.append(S.RigidObject(S.SHAPE_SPHERE, (0.004, -0.002, 0.003), (0.0125, 0, 0)))
    sc.sources.append(S.GaussianSource((-0.018, 0.012, 0.02), 2e-5))
    sc.listeners = np.array([[0.021, 0.011, -0.024], [-0.02, -0.015, 0.03], [0.016, -0.014, 0.0]])
    return sc


def test_grid_geometry_and_pml_counts(oracle_lib):
    sc = S.config1()
    o = oracle_lib.OracleSolver(sc)
    assert o.n_cells == 64 ** 3
    assert o.n_pml_cells == 176960          # 67 % of the cells for a 10-cell PML
    assert sc.n_pml_cells() == 176960
    assert S.config2().n_pml_cells() == 5537792


def test_pml_flags_match_width(oracle_lib):
    sc = small_scene(with_sphere=False)
    o = oracle_lib.OracleSolver(sc)
    flags, faces = o.classification()
    f = flags.reshape(sc.divisions)
    pml = (f & S.CELL_PML) > 0
    W = 4
    idx = np.indices(sc.divisions)
    expect = np.zeros(sc.divisions, dtype=bool)
    for d in range(3):
        expect |= (idx[d] < W) | (idx[d] >= sc.divisions[d] - W)
    assert np.array_equal(pml, expect)
    assert len(faces) == 0 and np.all(f & S.CELL_BULK)


def test_mls_reproduces_linear_fields(oracle_lib):
    rng = np.random.default_rng(0)
    p = np.array([0.01, -0.02, 0.005])
    pts = p + rng.uniform(-0.006, 0.006, size=(11, 3))
    a, g = 0.37, np.array([2.5, -1.25, 0.75])
    vals = a + (pts - p) @ g
    assert abs(oracle_lib.mls_c0(p, pts, vals) - a) < 1e-14


def test_ghost_faces_of_sphere(oracle_lib):
    sc = small_scene()
    o = oracle_lib.OracleSolver(sc)
    flags, faces = o.classification()
    solid = (flags & S.CELL_BULK) == 0
    ghost = (flags & S.CELL_GHOST) > 0
    assert ghost.sum() > 0 and np.all(solid[ghost])
    assert np.array_equal(np.unique(faces["owner_cell"]), np.nonzero(ghost)[0])
    # Szudzik key of (min, max) and neighbour = owner +- stride of the topology axis
    N = sc.divisions
    strides = {1: N[1] * N[2], 2: N[2], 3: 1}
    for f in faces[:50]:
        a, b = sorted((int(f["owner_cell"]), int(f["neighbour_cell"])))
        assert f["key"] == (a * a + a + b if a >= b else a + b * b)
        t = int(f["topology"])
        assert f["neighbour_cell"] == f["owner_cell"] + (1 if t > 0 else -1) * strides[abs(t)]
        assert flags[f["neighbour_cell"]] & S.CELL_BULK


def test_source_linearity_is_exact(oracle_lib):
    sc1 = small_scene()
    sc2 = small_scene()
    c0 = 1.0 / (math.sqrt(2.0 * math.pi) * sc1.sound_speed * 2e-5) ** 3
    sc1.sources[0].normalize_constant = c0
    sc2.sources[0].normalize_constant = 2.0 * c0
    y1 = oracle_lib.OracleSolver(sc1).step(30)
    y2 = oracle_lib.OracleSolver(sc2).step(30)
    assert np.array_equal(2.0 * y1, y2)


def test_mirror_symmetry_without_objects(oracle_lib):
    h = 0.005
    sc = S.Scene(cell_size=h, divisions=(20, 20, 20), time_step=S.reference_time_step(h), pml_width=4)
    sc.sources.append(S.GaussianSource((0.0, 0.0, 0.0), 2e-5))
    o = oracle_lib.OracleSolver(sc)
    o.step(40)
    p = o.field(S.FIELD_PRESSURE).reshape(20, 20, 20)
    assert np.abs(p).max() > 0
    for ax in range(3):
        assert np.allclose(p, np.flip(p, axis=ax), rtol=1e-12, atol=1e-12 * np.abs(p).max())
    assert np.allclose(p, p.transpose(1, 0, 2), rtol=1e-12, atol=1e-12 * np.abs(p).max())


def test_oracle_matches_numpy_restatement(oracle_lib):
    from tests.golden.numpy_fdtd import NumpyFDTD
    sc = small_scene()
    o = oracle_lib.OracleSolver(sc)
    npf = NumpyFDTD(sc)
    yo = o.step(sc.steps)
    yn = np.array([npf.step() for _ in range(sc.steps)])
    assert rel_l2(yo, yn) < 1e-11
    for which, arr in ((S.FIELD_PRESSURE, npf.p_cur), (S.FIELD_PRESSURE_PREV, npf.p_prev),
                       (S.FIELD_PML_PX, npf.pd[0]), (S.FIELD_VY, npf.v[1])):
        assert rel_l2(o.field(which), arr.reshape(-1)) < 1e-11, which
    fo, _ = o.classification()
    assert np.array_equal((fo & S.CELL_BULK) > 0, npf.bulk.reshape(-1))


def test_oracle_matches_golden_fixture(oracle_lib):
    path = os.path.join(HERE, "golden", "oracle_small.npz")
    g = np.load(path)
    sc = small_scene()
    y = oracle_lib.OracleSolver(sc).step(sc.steps)
    assert np.array_equal(y, g["listeners"])
    assert abs(float(g["numpy_rel_l2"])) < 1e-11


def test_translating_sphere_dipole_known_answer(oracle_lib):
    """The reference's analytic acceleration-noise solution for a rigidly
    accelerating sphere (AccelerationNoiseVibrationalSource.cpp:134-162):
    p(x,t) = rho a^3 cos(theta) / (2 c r) * da/dt(t - r/c) in the far field."""
    h = 0.004
    n = 48
    sc = S.Scene(cell_size=h, divisions=(n, n, n), time_step=S.reference_time_step(h), pml_width=8)
    R, A, tau = 0.02, 1.0e3, 1.0e-4
    t0 = 4 * tau
    sc.objects.append(S.RigidObject(S.SHAPE_SPHERE, (0.0, 0.0, 0.0), (R, 0, 0),
                                    accel_kind=S.ACCEL_GAUSSIAN_TRANSLATION, accel_amplitude=A,
                                    accel_t0=t0, accel_tau=tau, accel_dir=(0.0, 0.0, 1.0)))
    r = 0.052
    sc.listeners = np.array([[0.0, 0.0, r], [0.0, 0.0, -r], [r, 0.0, 0.0]])
    steps = 400
    y = oracle_lib.OracleSolver(sc).step(steps)
    t = (np.arange(steps) + 1) * sc.time_step
    ret = t - r / sc.sound_speed
    u = (ret - t0) / tau
    adot = A * np.exp(-u * u / 2.0) * (-u / tau)
    p_far = sc.density * R ** 3 / (2.0 * sc.sound_speed * r) * adot
    near = sc.density * R ** 3 / (2.0 * r * r) * A * np.exp(-u * u / 2.0)   # 1/r^2 term of the dipole
    p_ref = p_far + near
    on = y[:, 0]
    corr = np.dot(on, p_ref) / (np.linalg.norm(on) * np.linalg.norm(p_ref))
    assert corr > 0.9
    assert 0.6 < np.abs(on).max() / np.abs(p_ref).max() < 1.6
    # antisymmetric along the acceleration axis, ~zero broadside
    assert np.allclose(y[:, 0], -y[:, 1], atol=0.05 * np.abs(on).max())
    assert np.abs(y[:, 2]).max() < 0.05 * np.abs(on).max()


@pytest.mark.parametrize("preset,pml", [(1, 4.0), (2, 4.0), (0, 1.0), (0, 0.0)])
def test_oracle_engquist_matches_numpy_restatement(oracle_lib, preset, pml):
    """Sides without PML (wall presets, thin PML): the Engquist-Majda cells, the
    exterior values written into the current buffer and the untouched edge
    cells of three rotating buffers, against the numpy restatement."""
    from tests.golden.numpy_fdtd import NumpyFDTD
    h = 0.005
    sc = S.Scene(cell_size=h, divisions=(22, 20, 24), time_step=S.reference_time_step(h), pml_width=pml, steps=90)
    sc.boundary_condition_preset = preset
    sc.objects.append(S.RigidObject(S.SHAPE_SPHERE, (0.004, -0.003, 0.0), (0.012, 0, 0)))
    sc.sources.append(S.GaussianSource((0.02, 0.015, 0.025), 5e-5))
    sc.listeners = np.array([[-0.02, 0.02, -0.02], [0.0475, 0.01, 0.0], [0.01, -0.01, 0.0525]])
    o = oracle_lib.OracleSolver(sc)
    npf = NumpyFDTD(sc)
    assert npf.eng.any()
    yo = o.step(sc.steps)
    yn = np.array([npf.step() for _ in range(sc.steps)])
    assert np.abs(yo).max() > 0
    assert rel_l2(yo, yn) < 1e-11, rel_l2(yo, yn)
    assert rel_l2(o.field(S.FIELD_PRESSURE), npf.p_cur.reshape(-1)) < 1e-11
    assert rel_l2(o.field(S.FIELD_PRESSURE_PREV), npf.p_prev.reshape(-1)) < 1e-11
