"""FetchCell and SampleAxisAlignedSlice (PML_WaveSolver.cpp:439-458,
MAC_Grid.cpp:1941-1963) through the C-ABI against the oracle's restatement of
MAC_Grid::GetCell (MAC_Grid.cpp:4182-4258): geometry, cell type and flags
bit-exact, pressures, split pressures, face velocities, ghost-face pressures
and the stored Laplacian within the path's tolerance."""
import ctypes as C

import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200._lib import FDTDError
from acoustics_b200.solver import PML_WaveSolver
from tests.test_gpu_paths import moving_scene

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_FC64 = 1e-11  # the coupled solves stop at one machine epsilon
TOL_FP32 = 1e-4

EXACT = ("index", "indices", "n_gc_value", "r_identity", "centroid", "lower_corner", "upper_corner", "h")
VALUES = ("p_full", "p_directional", "vx", "vy", "vz", "gc_value")


def scene(alpha=0.0, fully_coupled=False):
    sc = S.config1(divisions=(40, 36, 44), pml_width=6, radius=0.03)
    sc.objects.append(S.RigidObject(S.SHAPE_BOX, (0.04, -0.04, 0.02), (0.02, 0.015, 0.01),
                                    accel_kind=S.ACCEL_GAUSSIAN_TRANSLATION, accel_amplitude=1e3,
                                    accel_t0=2e-4, accel_tau=8e-5, accel_dir=(0.6, 0.8, 0.0)))
    sc.air_viscosity_alpha = alpha
    if fully_coupled:
        sc.boundary_handling = S.BOUNDARY_FULLY_COUPLED
    return sc


def oracle_cells(o, index):
    return np.array([o.fetch_cell(int(i)) for i in index], dtype=S.CELL_DTYPE)


def close(a, b, tol):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    scale = max(float(np.abs(b).max()), 1e-300)
    return float(np.abs(a - b).max()) <= tol * scale


def compare(g, o, tol, values=VALUES, laplacian=True):
    for k in EXACT:
        assert np.array_equal(g[k], o[k]), k
    assert np.array_equal(g["flags"] & 0xFF, o["flags"] & 0xFF)
    for k in values:
        if k == "gc_value":  # -1 marks a missing face; the values are relative to the faces'
            face = o[k] != -1.0
            assert np.array_equal(g[k] != -1.0, face)
            assert not face.any() or close(g[k][face], o[k][face], tol), k
        else:
            assert close(g[k], o[k], tol), k
    if laplacian:
        has = (g["flags"] & S.CELLINFO_LAPLACIAN) != 0
        assert np.all(np.isnan(g["laplacian"][~has]))
        if has.any():
            # the 7-point Laplacian scales pressure differences by 1/h^2: its
            # rounding is relative to 12 max|p| / h^2, not to its own size
            x, y = g["laplacian"][has], o["laplacian"][has]
            scale = max(float(np.abs(y).max()), 12.0 * float(np.abs(o["p_full"]).max()) / float(o["h"][0]) ** 2)
            assert float(np.abs(x - y).max()) <= tol * scale
        return has
    return None


def slices(g, o, sc):
    """Slices through the bodies and through the PML along every axis, each
    against the oracle's cells of the same plane in the same order."""
    N = sc.divisions
    h = sc.cell_size
    lo = -0.5 * np.asarray(N) * h
    for dim in range(3):
        for off in (0.0, 0.04 if dim == 0 else -0.04, lo[dim] + 2.3 * h):
            cells = g.SampleAxisAlignedSlice(dim, off)
            d1, d2 = (dim + 1) % 3, (dim + 2) % 3
            assert cells.size == N[d1] * N[d2]
            k = min(int((off - (lo[dim] - h / 2)) / h), N[dim] - 1)
            assert np.all(cells["indices"][:, dim] == k)
            idx = np.zeros((N[d1], N[d2], 3), dtype=np.int64)
            idx[..., dim] = k
            idx[..., d1] = np.arange(N[d1])[:, None]
            idx[..., d2] = np.arange(N[d2])[None, :]
            flat = ((idx[..., 0] * N[1] + idx[..., 1]) * N[2] + idx[..., 2]).ravel()
            assert np.array_equal(cells["index"], flat)
            yield cells, oracle_cells(o, flat)


def ghost_and_pml_cells(o, n=64):
    flags, _ = o.classification()
    ghosts = np.nonzero((flags & S.CELL_GHOST) != 0)[0]
    pml = np.nonzero((flags & S.CELL_PML) != 0)[0]
    rng = np.random.default_rng(5)
    return np.concatenate([ghosts[:: max(1, ghosts.size // n)], rng.choice(pml, n, replace=False)])


def test_fetch_before_first_step(oracle_lib, fdtd_lib):
    sc = scene()
    o, g = oracle_lib.OracleSolver(sc), PML_WaveSolver(sc)
    idx = ghost_and_pml_cells(o)
    a = np.array([g.FetchCell(int(i)) for i in idx], dtype=S.CELL_DTYPE)
    b = oracle_cells(o, idx)
    has = compare(a, b, 0.0)
    assert has.all() and np.all(a["laplacian"] == 0.0)
    ghost = a["n_gc_value"] == 6
    assert ghost.any()
    assert np.all((a["gc_value"][ghost] == 0.0) | (a["gc_value"][ghost] == -1.0))
    assert np.all(a["gc_value"][~ghost] == -1.0)


@pytest.mark.parametrize("alpha", [0.0, 2e-5])
def test_fetch_fp64_fused(oracle_lib, fdtd_lib, alpha):
    sc = scene(alpha)
    o, g = oracle_lib.OracleSolver(sc), PML_WaveSolver(sc)
    o.step(90)
    g.step(90)
    n_ghost_faces = 0
    for a, b in slices(g, o, sc):
        has = compare(a, b, TOL_FP64)
        pml = (a["flags"] & S.CELL_PML) != 0
        # the fused kernels keep the Laplacian only with air viscosity, outside the PML
        assert np.array_equal(has, ~pml if alpha > 0 else np.zeros_like(has))
        n_ghost_faces += int(np.sum(a["gc_value"] != -1.0))
    assert n_ghost_faces > 0
    idx = ghost_and_pml_cells(o)
    a = np.array([g.FetchCell(int(i)) for i in idx], dtype=S.CELL_DTYPE)
    compare(a, oracle_cells(o, idx), TOL_FP64)
    assert np.all(a["flags"] & S.CELLINFO_PML_STATE)
    ghost = a["n_gc_value"] == 6
    assert np.abs(a["gc_value"][ghost][a["gc_value"][ghost] != -1.0]).max() > 0.0


def test_fetch_fp64_phased_viscosity(oracle_lib, fdtd_lib):
    """The phased path keeps the reference's Laplacian on every cell."""
    sc = scene(2e-5)
    o, g = oracle_lib.OracleSolver(sc), PML_WaveSolver(sc, kernel=S.KERNEL_PHASED)
    o.step(60)
    g.step(60)
    for a, b in slices(g, o, sc):
        has = compare(a, b, TOL_FP64)
        assert has.all()


def test_fetch_fully_coupled(oracle_lib, fdtd_lib):
    sc = scene(fully_coupled=True)
    o, g = oracle_lib.OracleSolver(sc), PML_WaveSolver(sc)
    o.step(80)
    g.step(80)
    idx = ghost_and_pml_cells(o, 200)
    a = np.array([g.FetchCell(int(i)) for i in idx], dtype=S.CELL_DTYPE)
    compare(a, oracle_cells(o, idx), TOL_FC64)


@pytest.mark.parametrize("pml_state", [S.PML_STATE_FULL, S.PML_STATE_AUTO])
def test_fetch_fp32(oracle_lib, fdtd_lib, pml_state):
    sc = scene()
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc, precision=S.PRECISION_FP32_COMPENSATED, pml_state=pml_state)
    o.step(90)
    g.step(90)
    reduced = g.pml_state() == S.PML_STATE_AUTO
    assert reduced == (pml_state == S.PML_STATE_AUTO)
    values = ("p_full", "gc_value") if reduced else VALUES
    for a, b in slices(g, o, sc):
        compare(a, b, TOL_FP32, values=values)
        held = (a["flags"] & S.CELLINFO_PML_STATE) != 0
        assert np.all(held != reduced)
        if reduced:
            assert np.all(np.isnan(a["p_directional"])) and np.all(np.isnan(a["vx"]))


def test_fetch_moving_bodies(oracle_lib, fdtd_lib):
    sc = moving_scene(steps=60)
    o, g = oracle_lib.OracleSolver(sc), PML_WaveSolver(sc)
    o.step(60)
    g.step(60)
    for a, b in slices(g, o, sc):
        has = compare(a, b, TOL_FP64)
        assert not has.any()


def test_fetch_arguments(fdtd_lib):
    sc = scene()
    g = PML_WaveSolver(sc)
    N = sc.divisions
    h = sc.cell_size
    lo = -0.5 * N[0] * h
    for bad in (-1, g.n_cells):
        with pytest.raises(FDTDError) as e:
            g.FetchCell(bad)
        assert e.value.status == -1
    with pytest.raises(FDTDError):
        g.SampleAxisAlignedSlice(3, 0.0)
    # the face grid starts half a cell below the cells; (int) truncates toward zero
    assert np.all(g.SampleAxisAlignedSlice(0, lo - h / 2)["indices"][:, 0] == 0)
    assert np.all(g.SampleAxisAlignedSlice(0, lo - 1.4 * h)["indices"][:, 0] == 0)
    assert np.all(g.SampleAxisAlignedSlice(0, lo + 100 * h)["indices"][:, 0] == N[0] - 1)
    with pytest.raises(FDTDError):
        g.SampleAxisAlignedSlice(0, lo - 1.6 * h)
    # count query, then a buffer one cell short
    n = C.c_int64(0)
    assert fdtd_lib.fdtd_solver_sample_slice(g._h, 1, C.c_double(0.0), None, 0, C.byref(n)) == 0
    assert n.value == N[2] * N[0]
    buf = np.zeros(n.value, dtype=S.CELL_DTYPE)
    assert fdtd_lib.fdtd_solver_sample_slice(g._h, 1, C.c_double(0.0), buf.ctypes.data, n.value - 1,
                                             C.byref(n)) == -1


def test_solver_domain(fdtd_lib):
    """GetSolverDomain: the grid's box, consistent with the cells' corners."""
    sc = scene()
    g = PML_WaveSolver(sc)
    lo, hi = g.GetSolverDomain()
    N, h = np.asarray(sc.divisions), sc.cell_size
    assert np.array_equal(lo, -(h * N) / 2.0)
    assert np.allclose(hi, lo + h * N, rtol=0, atol=1e-15)
    first = g.FetchCell(0)
    last = g.FetchCell(g.n_cells - 1)
    assert np.allclose(first["lower_corner"], lo, rtol=0, atol=1e-15)
    assert np.allclose(last["upper_corner"], hi, rtol=0, atol=1e-15)
