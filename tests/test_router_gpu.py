"""The request router with two solve servers (both on device 0 here: every
gpurun box has one GPU; the servers share nothing): requests spread over both
and every series equals a standalone solve's."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.router import ServerRouter
from acoustics_b200.solver import PML_WaveSolver

pytestmark = pytest.mark.gpu

P32 = S.PRECISION_FP32_COMPENSATED


def test_router_two_servers(fdtd_lib):
    rng = np.random.default_rng(61)
    scenes = [S.random_scene(rng, 28, 56, 3, 3, 60, 140, f"r{i}", pml=6) for i in range(6)]
    with ServerRouter(devices=[0, 0], precision=P32, graph_steps=8, chunk_steps=16) as r:
        keys = [r.submit(sc) for sc in scenes]
        assert {k[0] for k in keys} == {0, 1}
        for k, sc in zip(keys, scenes):
            y, _ = r.result(k)
            with PML_WaveSolver(sc, precision=P32) as g:
                assert np.array_equal(y, g.step(sc.steps))
        assert all(abs(w) < 1e-6 for w in r.work)
