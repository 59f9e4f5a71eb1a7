import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    # tuned tile shapes of this session only (the autotuner runs on a cache miss)
    if "FDTD_TUNE_CACHE" not in os.environ:
        import tempfile
        os.environ["FDTD_TUNE_CACHE"] = os.path.join(tempfile.mkdtemp(prefix="fdtd_tune_"), "tuned.json")
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import loader
    loader.build()
    loader.set_threads(os.cpu_count() or 1)
    return loader


@pytest.fixture(scope="session")
def fdtd_lib():
    from acoustics_b200 import build as b
    b.build()
    from acoustics_b200 import _lib
    return _lib.load()
