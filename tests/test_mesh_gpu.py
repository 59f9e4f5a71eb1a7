"""Triangle-mesh bodies on the GPU against the FP64 oracle: classification
bit-exact (flags and every ghost face), listener series within the FP64 / FP32
tolerances, static and moving (fresh cells interpolated through the mesh's
closest-point reflection)."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.solver import PML_WaveSolver
from tests._util import rel_l2

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_FP32 = 1e-4


def rot_z(deg):
    a = np.deg2rad(deg)
    return (np.cos(a), -np.sin(a), 0.0, np.sin(a), np.cos(a), 0.0, 0.0, 0.0, 1.0)


def mesh_scene(moving=False, steps=160):
    h = 0.004
    sc = S.Scene(cell_size=h, divisions=(48, 40, 40), time_step=S.reference_time_step(h), pml_width=6, steps=steps,
                 name="meshes_small")
    k = sc.time_step
    sc.meshes = [S.icosphere(0.014, 2), S.box_mesh((0.01, 0.007, 0.008))]
    sc.objects.append(S.RigidObject(S.SHAPE_MESH, (-0.031, 0.002, -0.001), (0, 0, 0), mesh=0,
                                    accel_kind=S.ACCEL_GAUSSIAN_TRANSLATION, accel_amplitude=1e3,
                                    accel_t0=30 * k, accel_tau=8 * k, accel_dir=(0, 0, 1)))
    box = S.RigidObject(S.SHAPE_MESH, (0.034, 0.006, 0.0015), (0, 0, 0), rotation=rot_z(25), mesh=1)
    if moving:
        box.motion = S.MOTION_BALLISTIC
        box.velocity = (-60.0, 0.0, 0.0)
        box.gravity = (0.0, 0.0, -9.81)
    sc.objects.append(box)
    sc.sources.append(S.GaussianSource((0.0, 0.04, 0.0), 5e-5))
    sc.listeners = np.array([[0.0, -0.03, 0.01], [0.02, 0.02, -0.02], [-0.04, 0.0, 0.03]])
    return sc


@pytest.mark.parametrize("moving", [False, True])
@pytest.mark.parametrize("precision,tol", [(S.PRECISION_FP64, TOL_FP64), (S.PRECISION_FP32_COMPENSATED, TOL_FP32)])
def test_meshes_match_oracle(oracle_lib, fdtd_lib, moving, precision, tol):
    sc = mesh_scene(moving)
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc, precision=precision)
    for chunk in range(4):
        yo, yg = o.step(40), g.step(40)
        assert rel_l2(yg, yo) <= tol, chunk
        fo, go = o.classification()
        fg, gg = g.GetGrid()
        assert np.array_equal(fo, fg), chunk
        assert np.array_equal(go, gg), chunk
    assert np.abs(yo).max() > 0


def test_box_mesh_classifies_like_the_analytic_box(fdtd_lib):
    """The exact mesh distance of a box surface is the analytic box's: the same
    pose (off the grid) gives the same classification and listener series."""
    def scene(as_mesh):
        h = 0.004
        sc = S.Scene(cell_size=h, divisions=(40, 40, 40), time_step=S.reference_time_step(h), pml_width=6,
                     steps=80, name="box_vs_mesh")
        half = (0.0123, 0.0071, 0.0094)
        pose = dict(rotation=rot_z(17), accel_kind=S.ACCEL_GAUSSIAN_TRANSLATION, accel_amplitude=1e3,
                    accel_t0=20 * sc.time_step, accel_tau=6 * sc.time_step, accel_dir=(1, 0, 0))
        if as_mesh:
            sc.meshes = [S.box_mesh(half)]
            sc.objects.append(S.RigidObject(S.SHAPE_MESH, (0.0011, -0.0023, 0.0007), (0, 0, 0), mesh=0, **pose))
        else:
            sc.objects.append(S.RigidObject(S.SHAPE_BOX, (0.0011, -0.0023, 0.0007), half, **pose))
        sc.sources.append(S.GaussianSource((0.0, 0.04, 0.0), 5e-5))
        sc.listeners = np.array([[0.0, -0.035, 0.01], [0.03, 0.02, -0.02]])
        return sc
    a = PML_WaveSolver(scene(False))
    m = PML_WaveSolver(scene(True))
    ya, ym = a.step(80), m.step(80)
    fa, ga = a.GetGrid()
    fm, gm = m.GetGrid()
    assert np.array_equal(fa, fm)
    assert np.array_equal(ga, gm)
    assert rel_l2(ym, ya) <= TOL_FP64


def test_mesh_members_in_batch_and_server(fdtd_lib):
    """A static mesh scene batched with analytic ones, and served through the
    solve server (which keeps its own copy of the mesh arrays): the series
    equal a standalone solver's bit for bit."""
    from acoustics_b200.batch import SolveBatch
    from acoustics_b200.server import SolveServer
    P32 = S.PRECISION_FP32_COMPENSATED
    mesh = mesh_scene(False, steps=60)
    rng = np.random.default_rng(11)
    others = [S.random_scene(rng, 28, 48, 3, 4, 40, 80, f"a{i}", pml=6) for i in range(3)]

    def alone(sc):
        with PML_WaveSolver(sc, precision=P32) as g:
            return g.step(sc.steps)

    with SolveBatch([others[0], mesh, others[1]], precision=P32, graph_steps=8) as b:
        b.run()
        for m, sc in enumerate([others[0], mesh, others[1]]):
            assert np.array_equal(b.output(m), alone(sc)), f"member {m}"
    with SolveServer(precision=P32, graph_steps=8, chunk_steps=16) as srv:
        ids = [srv.submit(others[2])]
        im = srv.submit(mesh)
        y, _ = srv.result(im)
        for i in ids:
            srv.result(i)
    assert np.array_equal(y, alone(mesh))


def test_concave_moving_mesh_matches_oracle(oracle_lib, fdtd_lib):
    """An extruded L (concave edges and vertices) crossing the grid: fresh cells
    through the mesh reflection, classification bit-exact after every chunk."""
    from tests.test_mesh_cpu import l_prism
    h = 0.004
    sc = S.Scene(cell_size=h, divisions=(44, 40, 36), time_step=S.reference_time_step(h), pml_width=6, steps=120,
                 name="l_prism_moving")
    m = l_prism(0.012)
    m.vertices = m.vertices - m.vertices.mean(axis=0)
    sc.meshes = [m]
    sc.objects.append(S.RigidObject(S.SHAPE_MESH, (0.01, -0.004, 0.002), (0, 0, 0), rotation=rot_z(20), mesh=0,
                                    motion=S.MOTION_BALLISTIC, velocity=(-50.0, 15.0, 0.0)))
    sc.sources.append(S.GaussianSource((0.0, 0.04, 0.0), 5e-5))
    sc.listeners = np.array([[0.0, -0.03, 0.01], [0.025, 0.02, -0.02]])
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc)
    for chunk in range(3):
        yo, yg = o.step(40), g.step(40)
        assert rel_l2(yg, yo) <= TOL_FP64, chunk
        fo, go = o.classification()
        fg, gg = g.GetGrid()
        assert np.array_equal(fo, fg), chunk
        assert np.array_equal(go, gg), chunk
