"""The autotuner on the GPU: it times every candidate shape, caches the
fastest for the grid class, SolveBatch picks the cached shape by default, and
the tuned shape changes no result bit (against an explicitly shaped batch and
against standalone solvers)."""
import numpy as np
import pytest

from acoustics_b200 import autotune as A
from acoustics_b200 import scene as S
from acoustics_b200.batch import SolveBatch
from acoustics_b200.solver import PML_WaveSolver

pytestmark = pytest.mark.gpu

P32 = S.PRECISION_FP32_COMPENSATED


def test_tuned_shape_is_cached_used_and_exact(fdtd_lib, tmp_path, monkeypatch):
    monkeypatch.setenv("FDTD_TUNE_CACHE", str(tmp_path / "tuned.json"))
    rng = np.random.default_rng(51)
    scenes = [S.random_scene(rng, 36, 64, 3, 4, 80, 140, f"t{i}", pml=6) for i in range(6)]
    e = A.tune(scenes, P32, sample=4, steps=16, candidates=[(2, 8), (4, 4), (8, 16)])
    assert set(e["timings_ms"]) == {"2x8", "4x4", "8x16"}
    assert all(v > 0 for v in e["timings_ms"].values())
    best = (e["x_chunk"], e["tile_y"])
    assert A.lookup(scenes, P32, A.device_name(0)) == best
    with SolveBatch(scenes, precision=P32, graph_steps=8) as b:
        assert b.shape == best
        b.run()
        tuned = [b.output(m) for m in range(len(scenes))]
    with SolveBatch(scenes, precision=P32, graph_steps=8, x_chunk=2, tile_y=8) as b:
        b.run()
        plain = [b.output(m) for m in range(len(scenes))]
    for m, sc in enumerate(scenes):
        assert np.array_equal(tuned[m], plain[m])
        with PML_WaveSolver(sc, precision=P32) as g:
            assert np.array_equal(tuned[m], g.step(sc.steps))
