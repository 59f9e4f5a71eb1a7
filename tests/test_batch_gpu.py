"""Batched stepping of uneven static solves: every member's listener series is
identical to the one a standalone solver of the same scene produces (same
kernels, same order of arithmetic), members join and finish at their own steps,
and the number of launches per batched step does not grow with the members."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.batch import SolveBatch
from acoustics_b200.solver import PML_WaveSolver
from tests._util import rel_l2

pytestmark = pytest.mark.gpu


def uneven_scenes(seed, n, edge_lo=28, edge_hi=56, steps_lo=40, steps_hi=110):
    rng = np.random.default_rng(seed)
    return [S.random_scene(rng, edge_lo, edge_hi, 3, 4, steps_lo, steps_hi, f"u{i}", pml=6) for i in range(n)]


def alone(sc, precision, steps):
    with PML_WaveSolver(sc, precision=precision) as g:
        return g.step(steps)


@pytest.mark.parametrize("precision", [S.PRECISION_FP64, S.PRECISION_FP32_COMPENSATED])
@pytest.mark.parametrize("graph_steps", [0, 8])
def test_batch_members_equal_standalone(fdtd_lib, precision, graph_steps):
    scenes = uneven_scenes(11, 6)
    with SolveBatch(scenes, precision=precision, graph_steps=graph_steps) as b:
        b.run()
        for m, sc in enumerate(scenes):
            done, total, nl, st = b.info(m)
            assert (done, total, nl, st) == (sc.steps, sc.steps, sc.n_listeners, 0)
            y = b.output(m)
            assert y.shape == (sc.steps, sc.n_listeners)
            assert np.array_equal(y, alone(sc, precision, sc.steps)), f"member {m}"


@pytest.mark.parametrize("tile", [dict(x_chunk=2, tile_y=2), dict(x_chunk=8, tile_y=1), dict(x_chunk=4, tile_y=16)])
def test_batch_tile_shapes(fdtd_lib, tile):
    scenes = uneven_scenes(12, 4)
    with SolveBatch(scenes, precision=S.PRECISION_FP32_COMPENSATED, **tile) as b:
        b.run()
        for m, sc in enumerate(scenes):
            assert np.array_equal(b.output(m), alone(sc, S.PRECISION_FP32_COMPENSATED, sc.steps))


def test_batch_fp64_matches_oracle(oracle_lib, fdtd_lib):
    sc = uneven_scenes(13, 1)[0]
    with SolveBatch([sc], precision=S.PRECISION_FP64) as b:
        b.run()
        y = b.output(0)
    yo = oracle_lib.OracleSolver(sc).step(sc.steps)
    assert rel_l2(y, yo) <= 1e-12


def test_members_join_mid_run_and_release(fdtd_lib):
    p = S.PRECISION_FP32_COMPENSATED
    first = uneven_scenes(14, 3)
    late = uneven_scenes(15, 2)
    with SolveBatch(first, precision=p, graph_steps=4) as b:
        assert b.step(23) == 3
        ids = [b.add(sc, sc.steps) for sc in late]
        while b.step(17) > 0:
            pass
        for m, sc in enumerate(first + late):
            assert np.array_equal(b.output(m), alone(sc, p, sc.steps)), f"member {m}"
        before = b.device_bytes()
        b.release(ids[0])
        assert b.device_bytes() < before
        with pytest.raises(Exception):
            b.output(ids[0])
        # the freed index is reused and the new member runs like a standalone solver
        again = late[1]
        assert b.add(again, 30) == ids[0]
        while b.step(64) > 0:
            pass
        assert np.array_equal(b.output(ids[0]), alone(again, p, 30))


def test_launches_per_step_do_not_grow_with_members(fdtd_lib):
    p = S.PRECISION_FP32_COMPENSATED
    counts = []
    for n in (2, 8):
        scenes = uneven_scenes(16, n, steps_lo=200, steps_hi=200)
        with SolveBatch(scenes, precision=p, graph_steps=0) as b:
            b.step(10)
            counts.append(b.last_launch_count() / 10)
    assert counts[0] == counts[1] <= 7


def test_moving_scene_is_refused(fdtd_lib):
    sc = S.config1(divisions=(40, 36, 32), pml_width=6, radius=0.02, steps=10)
    sc.objects[0].motion = S.MOTION_BALLISTIC
    sc.objects[0].velocity = (0.5, 0.0, 0.0)
    with SolveBatch([], precision=S.PRECISION_FP32_COMPENSATED) as b:
        with pytest.raises(Exception, match="UNSUPPORTED|moving"):
            b.add(sc, 10)


def test_batch_mixed_pml_states(fdtd_lib):
    """FP32 members with the reduced PML state and one with the full state (a
    box reaching into the PML) step in one batch; each equals its standalone solve."""
    scenes = uneven_scenes(21, 3)
    sc = S.config1(divisions=(40, 36, 44), pml_width=6, radius=0.02, steps=60)
    sc.objects.append(S.RigidObject(S.SHAPE_BOX, (0.08, 0.0, 0.0), (0.04, 0.02, 0.02)))
    scenes.insert(1, sc)
    p = S.PRECISION_FP32_COMPENSATED
    with PML_WaveSolver(sc, precision=p) as g:
        assert g.pml_state() == S.PML_STATE_FULL
    with PML_WaveSolver(scenes[0], precision=p) as g:
        assert g.pml_state() == S.PML_STATE_AUTO
    with SolveBatch(scenes, precision=p, graph_steps=8) as b:
        b.run()
        for m, s in enumerate(scenes):
            assert np.array_equal(b.output(m), alone(s, p, s.steps)), f"member {m}"
