"""FP64 CUDA path vs the FP64 CPU oracle through the C-ABI (configuration 1 and
small variants): classification bit-exact, listener series and fields within
1e-12 relative L2."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.solver import PML_WaveSolver

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)


def run_pair(oracle_lib, sc, steps, **kw):
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc, **kw)
    yo = o.step(steps)
    yg = g.step(steps)
    return o, g, yo, yg


def test_config1_listeners_fp64(oracle_lib, fdtd_lib):
    sc = S.config1()
    o, g, yo, yg = run_pair(oracle_lib, sc, 500)
    assert np.all(np.isfinite(yg))
    err = rel_l2(yg, yo)
    print("cfg1 fp64 listener rel L2", err, "max abs", np.abs(yg - yo).max())
    assert err <= TOL_FP64


def test_config1_classification_bitexact(oracle_lib, fdtd_lib):
    sc = S.config1()
    o, g, _, _ = run_pair(oracle_lib, sc, 3)
    fo, go = o.classification()
    fg, gg = g.GetGrid()
    assert np.array_equal(fo, fg)
    assert len(go) == len(gg)
    for k in ("owner_cell", "neighbour_cell", "topology", "type", "boundary_object", "key"):
        assert np.array_equal(go[k], gg[k]), k


def test_config1_fields_fp64(oracle_lib, fdtd_lib):
    sc = S.config1()
    o, g, _, _ = run_pair(oracle_lib, sc, 120)
    for which in (S.FIELD_PRESSURE, S.FIELD_PRESSURE_PREV, S.FIELD_PML_PX, S.FIELD_PML_PY, S.FIELD_PML_PZ):
        a, b = g.field(which), o.field(which)
        assert rel_l2(a, b) <= TOL_FP64, which
    for which in (S.FIELD_VX, S.FIELD_VY, S.FIELD_VZ):
        a, b = g.field(which), o.field(which)
        assert rel_l2(a, b) <= TOL_FP64, which
