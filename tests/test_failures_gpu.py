"""Failure paths, made on the host (no GPU fault): a NaN source amplitude gives
FDTD_ERR_NUMERIC from a solver and from a batch member; an injected device
allocation failure gives FDTD_ERR_OOM at creation, at a batch admission (the
batch keeps stepping its other members) and at a server admission (the other
requests complete); an injected host allocation failure gives FDTD_ERR_OOM
and the handle stays usable; a server wait with a short limit times out;
cancelled requests (queued and running) release their bytes; evicted members
resume from their snapshot and their series equal uninterrupted solves bit for
bit.  The reference raises exceptions in these places (MAC_Grid.cpp:2050-2053,
PML_WaveSolver.cpp:231-234) and has no server."""
import time

import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200._lib import FDTDError, load
from acoustics_b200.batch import SolveBatch, scene_device_bytes
from acoustics_b200.server import SolveServer
from acoustics_b200.solver import PML_WaveSolver

pytestmark = pytest.mark.gpu

P32 = S.PRECISION_FP32_COMPENSATED
NUMERIC, OOM, TIMEOUT, CANCELLED = (S.STATUS_CODE[k] for k in ("FDTD_ERR_NUMERIC", "FDTD_ERR_OOM",
                                                                 "FDTD_ERR_TIMEOUT", "FDTD_ERR_CANCELLED"))
INJ_NONE, INJ_DEVICE, INJ_HOST = 0, 1, 2


def scenes(seed, n, steps_lo=60, steps_hi=160, lo=28, hi=60):
    rng = np.random.default_rng(seed)
    return [S.random_scene(rng, lo, hi, 3, 4, steps_lo, steps_hi, f"f{seed}_{i}", pml=6) for i in range(n)]


def alone(sc, steps=None):
    with PML_WaveSolver(sc, precision=P32) as g:
        return g.step(steps or sc.steps)


@pytest.fixture(autouse=True)
def disarm():
    yield
    load().fdtd_debug_inject_failure(INJ_NONE, 0)


def nan_scene(late=False):
    sc = scenes(31, 1)[0]
    sc.sources[0].normalize_constant = float("nan")
    if late:
        # the time factor underflows to zero (the source is off) for the first ~60 steps
        sc.sources[0].offset_time = 40 * sc.sources[0].width_time
    # a listener on the source: the NaN reaches it at once
    sc.listeners = np.vstack([np.asarray(sc.sources[0].position)[None, :], sc.listeners])
    return sc


@pytest.mark.parametrize("precision", [S.PRECISION_FP64, P32])
def test_nan_source_amplitude_is_numeric_error(fdtd_lib, precision):
    with PML_WaveSolver(nan_scene(), precision=precision) as g:
        with pytest.raises(FDTDError) as e:
            g.step(40)
        assert e.value.status == NUMERIC


def test_nan_source_in_batch_member(fdtd_lib):
    good = scenes(32, 2)
    with SolveBatch([good[0], nan_scene(late=True), good[1]], precision=P32, graph_steps=8) as b:
        b.run()
        assert b.info(1)[3] == NUMERIC
        with pytest.raises(FDTDError):
            b.output(1)
        for m, sc in ((0, good[0]), (2, good[1])):
            assert b.info(m)[3] == 0
            assert np.array_equal(b.output(m), alone(sc))


def test_injected_device_allocation_failure(fdtd_lib):
    L = load()
    a, c = scenes(33, 2)
    assert L.fdtd_debug_inject_failure(INJ_DEVICE, 0) == 0
    with pytest.raises(FDTDError) as e:
        PML_WaveSolver(a, precision=P32)
    assert e.value.status == OOM
    PML_WaveSolver(a, precision=P32).close()  # the next creation succeeds
    # a batch admission fails; the batch keeps stepping its member
    with SolveBatch([a], precision=P32, graph_steps=8) as b:
        b.step(20)
        L.fdtd_debug_inject_failure(INJ_DEVICE, 0)
        with pytest.raises(FDTDError) as e:
            b.add(c, c.steps)
        assert e.value.status == OOM
        b.run()
        assert np.array_equal(b.output(0), alone(a))


def test_injected_failure_at_server_admission(fdtd_lib):
    L = load()
    reqs = scenes(34, 3)
    with SolveServer(precision=P32, graph_steps=8, chunk_steps=16, max_members=1) as srv:
        ids = [srv.submit(reqs[0])]
        L.fdtd_debug_inject_failure(INJ_DEVICE, 0)  # the next admission (request 1 or 2 is queued) fails
        ids += [srv.submit(reqs[1]), srv.submit(reqs[2])]
        outcomes = []
        for i, sc in zip(ids, reqs):
            try:
                y, _ = srv.result(i)
                assert np.array_equal(y, alone(sc))
                outcomes.append("done")
            except FDTDError as e:
                assert e.status == OOM
                outcomes.append("oom")
        assert outcomes.count("oom") == 1
        st = srv.stats()
        assert st["failed"] == 1 and st["completed"] == 2 and st["device_bytes_in_use"] == 0


def test_injected_host_allocation_failure_keeps_handle(fdtd_lib):
    L = load()
    sc = scenes(35, 1)[0]
    with PML_WaveSolver(sc, precision=P32) as g:
        y0 = g.step(30)
        L.fdtd_debug_inject_failure(INJ_HOST, 0)
        with pytest.raises(FDTDError) as e:
            g.field(S.FIELD_PRESSURE)
        assert e.value.status == OOM
        p = g.field(S.FIELD_PRESSURE)  # usable again
        assert np.isfinite(p).all()
        y1 = g.step(sc.steps - 30)
    assert np.array_equal(np.concatenate([y0, y1]), alone(sc))


def test_server_wait_timeout(fdtd_lib):
    sc = scenes(36, 1, steps_lo=3000, steps_hi=3000, lo=90, hi=100)[0]
    with SolveServer(precision=P32, graph_steps=8) as srv:
        rid = srv.submit(sc)
        with pytest.raises(FDTDError) as e:
            srv.wait(rid, 0.001)
        assert e.value.status == TIMEOUT
        srv.cancel(rid)
        srv.drain()


def _wait_running(srv, rid, min_steps=1, limit_s=60.0):
    t0 = time.time()
    while time.time() - t0 < limit_s:
        st, done, _ = srv.poll(rid)
        if st == S.REQ_RUNNING and done >= min_steps:
            return done
        time.sleep(0.002)
    raise AssertionError("request never ran")


def test_cancel_queued_and_running(fdtd_lib):
    long_a, long_b = scenes(37, 2, steps_lo=20000, steps_hi=20000, lo=95, hi=100)
    short = scenes(38, 1)[0]
    with SolveServer(precision=P32, graph_steps=8, chunk_steps=16, max_members=1) as srv:
        ia, ib, ic = srv.submit(long_a), srv.submit(long_b), srv.submit(short)
        _wait_running(srv, ia)
        srv.cancel(ib)                        # queued
        assert srv.poll(ib)[0] == S.REQ_CANCELLED
        srv.cancel(ia)                        # running: stopped after its chunk
        for rid in (ia, ib):
            with pytest.raises(FDTDError) as e:
                srv.result(rid)
            assert e.value.status == CANCELLED
        y, _ = srv.result(ic)
        assert np.array_equal(y, alone(short))
        with pytest.raises(FDTDError):
            srv.cancel(ic)                    # finished (and forgotten)
        st = srv.stats()
        assert st["cancelled"] == 2 and st["completed"] == 1 and st["device_bytes_in_use"] == 0


def test_eviction_resumes_bit_exact(fdtd_lib):
    big = scenes(39, 1, steps_lo=1500, steps_hi=1500, lo=70, hi=80)[0]
    small = scenes(40, 1, steps_lo=100, steps_hi=100, lo=40, hi=50)[0]
    nb, ns = scene_device_bytes(big), scene_device_bytes(small)
    assert ns < nb
    budget = nb + ns // 2                     # the two do not fit together
    with SolveServer(precision=P32, graph_steps=8, chunk_steps=16, hbm_budget_bytes=budget, preempt=True) as srv:
        ib = srv.submit(big)
        _wait_running(srv, ib, min_steps=100)
        i_s = srv.submit(small)               # evicts the big request, runs, and the big one resumes
        ys, _ = srv.result(i_s)
        yb, _ = srv.result(ib)
        st = srv.stats()
    assert st["evictions"] >= 1
    assert np.array_equal(ys, alone(small))
    assert np.array_equal(yb, alone(big))


def test_no_eviction_without_preempt(fdtd_lib):
    big = scenes(39, 1, steps_lo=600, steps_hi=600, lo=70, hi=80)[0]
    small = scenes(40, 1, steps_lo=100, steps_hi=100, lo=40, hi=50)[0]
    budget = scene_device_bytes(big) + scene_device_bytes(small) // 2
    with SolveServer(precision=P32, graph_steps=8, chunk_steps=16, hbm_budget_bytes=budget) as srv:
        ib = srv.submit(big)
        _wait_running(srv, ib)
        i_s = srv.submit(small)
        ys, _ = srv.result(i_s)
        yb, _ = srv.result(ib)
        assert srv.stats()["evictions"] == 0
    assert np.array_equal(yb, alone(big))
    assert np.array_equal(ys, alone(small))
