"""Regenerates tests/golden/oracle_small.npz: the FP64 oracle's listener series
for the small sphere scene of tests/test_oracle_cpu.py, together with its
relative L2 distance to the independent numpy restatement.

  python tests/golden/make_fixtures.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import loader  # noqa: E402
from tests.golden.numpy_fdtd import NumpyFDTD  # noqa: E402
from tests.test_oracle_cpu import small_scene  # noqa: E402


def main():
    loader.build()
    sc = small_scene()
    y = loader.OracleSolver(sc).step(sc.steps)
    npf = NumpyFDTD(sc)
    yn = np.array([npf.step() for _ in range(sc.steps)])
    err = np.linalg.norm(y - yn) / np.linalg.norm(yn)
    np.savez(os.path.join(HERE, "oracle_small.npz"), listeners=y, numpy_listeners=yn, numpy_rel_l2=err)
    print("oracle vs numpy rel L2", err)


if __name__ == "__main__":
    main()
