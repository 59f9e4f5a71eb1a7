"""Keyframed bodies (a box turning a quarter turn and a sphere moving on
keyframes, FDTD_RigidObject_Animator.cpp:128-155) against the FP64 oracle:
classification and every ghost-face record bit-exact after every step,
listener series within 1e-12 (FP64) and 1e-4 (FP32)."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.solver import PML_WaveSolver
from tests._util import rel_l2
from tests.test_kinematics_cpu import keyframed_scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(S.PRECISION_FP64, 1e-12), (S.PRECISION_FP32_COMPENSATED, 1e-4)])
def test_keyframed_bodies_against_oracle(oracle_lib, fdtd_lib, precision, tol):
    sc = keyframed_scene()
    o = oracle_lib.OracleSolver(sc)
    g = PML_WaveSolver(sc, precision=precision)
    yo, yg = [], []
    for n in range(sc.steps):
        yo.append(o.step(1))
        yg.append(g.step(1))
        fo, go = o.classification()
        fg, gg = g.GetGrid()
        assert np.array_equal(fo, fg), n
        assert np.array_equal(go, gg), n
    yo, yg = np.concatenate(yo), np.concatenate(yg)
    assert np.abs(yo).max() > 0
    assert rel_l2(yg, yo) <= tol
    assert rel_l2(g.field(S.FIELD_PRESSURE), o.field(S.FIELD_PRESSURE)) <= tol
