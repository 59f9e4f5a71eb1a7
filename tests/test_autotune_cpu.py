"""The tile-shape autotuner's cache and grid classes (host only)."""
import numpy as np

from acoustics_b200 import autotune as A
from acoustics_b200 import scene as S


def test_grid_class_buckets():
    rng = np.random.default_rng(5)
    small = [S.random_scene(rng, 48, 60, 2, 2, 10, 20, f"s{i}") for i in range(4)]
    large = [S.random_scene(rng, 140, 160, 2, 2, 10, 20, f"l{i}") for i in range(4)]
    f32 = S.PRECISION_FP32_COMPENSATED
    k1, k2 = A.grid_class(small, f32, "B200"), A.grid_class(large, f32, "B200")
    assert k1 != k2 and k1.startswith("fp32|B200|")
    assert A.grid_class(small, S.PRECISION_FP64, "B200").startswith("fp64|")
    assert A.grid_class(small, f32, "B200") == k1  # deterministic


def test_cache_roundtrip(tmp_path):
    path = str(tmp_path / "tuned.json")
    rng = np.random.default_rng(6)
    scenes = [S.random_scene(rng, 48, 60, 2, 2, 10, 20, f"s{i}") for i in range(3)]
    f32 = S.PRECISION_FP32_COMPENSATED
    assert A.lookup(scenes, f32, "B200", path) is None
    A.store(A.grid_class(scenes, f32, "B200"), {"x_chunk": 4, "tile_y": 16, "ms_per_step": 0.1}, path)
    assert A.lookup(scenes, f32, "B200", path) == (4, 16)
    assert A.lookup(scenes, f32, "H100", path) is None
    # a miss without tuning falls back to the defaults
    other = [S.random_scene(rng, 140, 150, 2, 2, 10, 20, "o")]
    assert A.shapes_for(other, f32, tune_on_miss=False, path=path) == A.DEFAULT_SHAPE


def test_sample_spans_sizes():
    rng = np.random.default_rng(7)
    scenes = [S.random_scene(rng, 30, 90, 2, 2, 10, 20, f"s{i}") for i in range(20)]
    smp = A._sample(scenes, 5, 200)
    assert 1 < len(smp) <= 5 and all(sc.steps == 200 for sc in smp)
    cells = sorted(sc.n_cells for sc in scenes)
    assert min(sc.n_cells for sc in smp) == cells[0] and max(sc.n_cells for sc in smp) == cells[-1]
