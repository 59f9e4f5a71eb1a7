"""Solve server (continuous batching): a request's series is the same alone and
mixed with other requests that arrive while it runs, and equals a standalone
solver's; admission respects the device-byte budget; FIFO service with one
member; statistics are consistent."""
import time

import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.batch import scene_device_bytes
from acoustics_b200.server import SolveServer
from acoustics_b200.solver import PML_WaveSolver
from tests._util import rel_l2

pytestmark = pytest.mark.gpu

P32 = S.PRECISION_FP32_COMPENSATED


def scenes(seed, n, steps_lo=60, steps_hi=160):
    rng = np.random.default_rng(seed)
    return [S.random_scene(rng, 28, 60, 4, 6, steps_lo, steps_hi, f"req{i}", pml=6) for i in range(n)]


def test_result_same_alone_and_mixed(fdtd_lib, oracle_lib):
    a, *others = scenes(21, 5)
    with SolveServer(precision=P32, graph_steps=8, chunk_steps=16) as srv:
        y_alone, _ = srv.result(srv.submit(a))
    with SolveServer(precision=P32, graph_steps=8, chunk_steps=16) as srv:
        ids = [srv.submit(others[0]), srv.submit(others[1])]
        time.sleep(0.02)  # A arrives while the first two run
        ia = srv.submit(a)
        ids += [srv.submit(others[2]), srv.submit(others[3])]
        y_mixed, _ = srv.result(ia)
        for i, sc in zip(ids, others):
            y, _ = srv.result(i)
            with PML_WaveSolver(sc, precision=P32) as g:
                assert np.array_equal(y, g.step(sc.steps))
        st = srv.stats()
        assert st["completed"] == 5 and st["failed"] == 0
        assert st["peak_members"] >= 2
    assert np.array_equal(y_alone, y_mixed)
    with PML_WaveSolver(a, precision=P32) as g:
        assert np.array_equal(y_mixed, g.step(a.steps))
    # FP32 compensated against the FP64 oracle
    yo = oracle_lib.OracleSolver(a).step(a.steps)
    assert rel_l2(y_mixed, yo) <= 1e-4


def test_admission_by_device_bytes(fdtd_lib):
    reqs = scenes(22, 6)
    need = [scene_device_bytes(sc, precision=P32) for sc in reqs]
    budget = int(2.2 * max(need))
    with SolveServer(precision=P32, hbm_budget_bytes=budget, chunk_steps=8) as srv:
        ids = [srv.submit(sc) for sc in reqs]
        srv.drain(timeout_s=120)
        st = srv.stats()
        assert st["completed"] == 6
        assert 0 < st["peak_device_bytes"] <= budget
        assert sum(need) > budget  # the budget did hold requests back
        assert st["peak_members"] <= budget // min(need)
        for i, sc in zip(ids, reqs):
            y, lat = srv.result(i)
            assert y.shape == (sc.steps, sc.n_listeners) and lat > 0
        big = S.config1(divisions=(96, 96, 96))
        with pytest.raises(Exception):
            srv.submit(big, 10)  # footprint above the whole budget


def test_fifo_with_one_member(fdtd_lib):
    reqs = scenes(23, 4)
    with SolveServer(precision=P32, max_members=1) as srv:
        ids = [srv.submit(sc) for sc in reqs]
        lats = [srv.result(i)[1] for i in ids]
        st = srv.stats()
    assert st["peak_members"] == 1
    assert lats == sorted(lats)  # served in arrival order
    assert st["p50_latency_s"] <= st["p99_latency_s"]
    assert st["solves_per_s"] > 0 and st["cell_steps_per_s"] > 0


def test_fp64_server_matches_standalone(fdtd_lib):
    reqs = scenes(24, 3)
    with SolveServer(precision=S.PRECISION_FP64, graph_steps=0) as srv:
        ids = [srv.submit(sc) for sc in reqs]
        for i, sc in zip(ids, reqs):
            y, _ = srv.result(i)
            with PML_WaveSolver(sc) as g:
                assert np.array_equal(y, g.step(sc.steps))
