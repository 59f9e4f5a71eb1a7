"""The reference's output files written from the GPU state: the end-of-run
snapshot (FDTD_AcousticSimulator::_SaveSimulationSnapshot) against the FP64
oracle's fields, a restart from it, the solver-config position files and the
per-step field dumps (x-fastest order)."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200._lib import FDTDError
from acoustics_b200.solver import PML_WaveSolver, read_matrix
from tests._util import rel_l2

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def scene():
    return S.config1(divisions=(36, 32, 40), pml_width=6, radius=0.02)


def test_snapshot_matches_oracle_fields(oracle_lib, fdtd_lib, tmp_path):
    sc = scene()
    n = 61
    o = oracle_lib.OracleSolver(sc)
    o.step(n)
    g = PML_WaveSolver(sc)
    g.step(n)
    pat = str(tmp_path / "run_%s")
    g.save_snapshot("3", pat)
    f = lambda name: read_matrix(pat.replace("%s", f"snapshot_3_{name}"))  # noqa: E731
    ind = int(open(pat.replace("%s", "snapshot_3_p_collocated_ind.dat")).read())
    assert ind == (1 + n) % 3
    N = sc.n_cells
    assert rel_l2(f(f"p_collocated_{ind}.dat").ravel(), o.field(S.FIELD_PRESSURE)) <= TOL_FP64
    assert rel_l2(f(f"p_collocated_{(ind + 2) % 3}.dat").ravel(), o.field(S.FIELD_PRESSURE_PREV)) <= TOL_FP64
    assert not f(f"p_collocated_{(ind + 1) % 3}.dat").any()
    assert f("p_pml_full.dat").shape == (N, 1) and not f("p_pml_full.dat").any()
    for d in range(3):
        assert rel_l2(f(f"p_pml_{d}.dat").ravel(), o.field(S.FIELD_PML_PX + d)) <= TOL_FP64
        v = f(f"v_pml_{d}.dat")
        assert v.shape[1] == 1
        assert rel_l2(v.ravel(), o.field(S.FIELD_VX + d)) <= TOL_FP64


@pytest.mark.parametrize("precision", [S.PRECISION_FP64, S.PRECISION_FP32_COMPENSATED])
def test_restart_from_snapshot(fdtd_lib, tmp_path, precision):
    """A solve reset to the snapshot's time and loaded from it continues as the
    original does."""
    sc = scene()
    kw = dict(precision=precision, pml_state=S.PML_STATE_FULL)
    a = PML_WaveSolver(sc, **kw)
    a.step(50)
    pat = str(tmp_path / "%s")
    a.save_snapshot("0", pat)
    t = a.time
    ya = a.step(40)
    b = PML_WaveSolver(sc, **kw)
    b.Reinitialize_PML_WaveSolver(t)
    b.load_snapshot("0", pat)
    yb = b.step(40)
    tol = TOL_FP64 if precision == S.PRECISION_FP64 else 1e-6
    assert rel_l2(yb, ya) <= tol


def test_snapshot_needs_the_full_pml_state(fdtd_lib, tmp_path):
    g = PML_WaveSolver(scene(), precision=S.PRECISION_FP32_COMPENSATED)
    assert g.pml_state() == S.PML_STATE_AUTO
    g.step(3)
    with pytest.raises(FDTDError):
        g.save_snapshot("0", str(tmp_path / "%s"))


def test_config_and_field_dumps(fdtd_lib, tmp_path):
    sc = scene()
    g = PML_WaveSolver(sc)
    g.step(20)
    pat = str(tmp_path / "out_%s")
    g.save_config(pat)
    nx, ny, nz = sc.divisions
    h = sc.cell_size
    pos = read_matrix(pat.replace("%s", "pressure_vertex_position.dat"))
    assert pos.shape == (nx * ny * nz, 3)
    lo = np.asarray(sc.domain_center) - h * np.asarray(sc.divisions) / 2
    assert np.allclose(pos[0], lo + 0.5 * h) and np.allclose(pos[1] - pos[0], [h, 0, 0])  # x fastest
    vx = read_matrix(pat.replace("%s", "velocity_0_vertex_position.dat"))
    assert vx.shape == ((nx + 1) * ny * nz, 3) and np.allclose(vx[0], lo + [0, 0.5 * h, 0.5 * h])
    lis = read_matrix(pat.replace("%s", "listening_position.dat"))
    assert np.allclose(lis, np.asarray(sc.listeners))
    p = str(tmp_path / "data_pressure_00000020.dat")
    g.save_field_timestep(p)
    dump = read_matrix(p).ravel()
    dense = g.field(S.FIELD_PRESSURE).reshape(nx, ny, nz)
    assert np.array_equal(dump, dense.transpose(2, 1, 0).ravel())
