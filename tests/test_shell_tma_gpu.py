"""The TMA-staged PML shell (3-D tensor copies of every plane into a
shared-memory ring, FDTD_SHELL_STAGING_TMA) against the per-thread cp.async
shell (the default) on the reduced PML state: the arithmetic per cell is the
same, so listener series and pressure fields must be equal bit for bit, on
grids whose edges and PML widths are not multiples of the kernel's windows;
with graphs it stays within 1e-4 of the FP64 oracle."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.solver import PML_WaveSolver
from tests._util import rel_l2, small_config2

pytestmark = pytest.mark.gpu

F32 = S.PRECISION_FP32_COMPENSATED


def _uneven(seed, pml):
    rng = np.random.default_rng(seed)
    return S.random_scene(rng, 37, 75, 3, 4, 90, 90, f"tma{seed}", pml=pml)


SCENES = {
    "config1_64cube_pml10": lambda: S.config1(),
    "config2_80cube_pml8": lambda: small_config2(),
    "config1_pml6.5": lambda: S.config1(divisions=(40, 36, 44), pml_width=6.5, radius=0.02),
    "uneven_pml6": lambda: _uneven(21, 6),
    "uneven_pml8": lambda: _uneven(22, 8),
    "uneven_pml5": lambda: _uneven(23, 5),
    "config2_128cube_pml8": lambda: S.config2(n=128),
    # long rows: the default kernel runs the plain-z columns on their own boxes
    "config2_192cube_pml12": lambda: S.config2(n=192),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_tma_shell_equals_ring_shell(fdtd_lib, name):
    sc = SCENES[name]()
    steps = 120
    ring = PML_WaveSolver(sc, precision=F32)
    tma = PML_WaveSolver(sc, precision=F32, shell_staging=S.SHELL_STAGING_TMA)
    assert ring.pml_state() == S.PML_STATE_AUTO
    assert ring.shell_staging() == S.SHELL_STAGING_RING
    assert tma.shell_staging() == S.SHELL_STAGING_TMA
    ya, yb = ring.step(steps), tma.step(steps)
    assert np.abs(ya).max() > 0
    assert np.array_equal(ya, yb)
    assert np.array_equal(ring.field(S.FIELD_PRESSURE), tma.field(S.FIELD_PRESSURE))
    assert np.array_equal(ring.field(S.FIELD_PRESSURE_PREV), tma.field(S.FIELD_PRESSURE_PREV))
    ring.close()
    tma.close()


def test_tma_shell_with_graphs_against_oracle(oracle_lib, fdtd_lib):
    sc = small_config2()
    yo = oracle_lib.OracleSolver(sc).step(sc.steps)
    g = PML_WaveSolver(sc, precision=F32, graph_steps=16, shell_staging=S.SHELL_STAGING_TMA)
    assert g.shell_staging() == S.SHELL_STAGING_TMA
    yg = g.step(sc.steps)
    assert rel_l2(yg, yo) <= 1e-4


def test_full_state_has_no_reduced_shell(fdtd_lib):
    assert PML_WaveSolver(S.config1()).shell_staging() == -1
    sc = S.config1()
    assert PML_WaveSolver(sc, precision=F32, pml_state=S.PML_STATE_FULL).shell_staging() == -1
