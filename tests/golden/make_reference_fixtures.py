"""Regenerates tests/golden/small_ball_mesh.npz from the reference project's own
fixture mesh work/meshes/small_ball/small_ball.obj (a closed sphere of radius
5 cm, 2562 vertices, 5120 triangles), read with the library's .obj reader, so
the GPU tests can run the reference's mesh where the reference tree is absent.

  python tests/golden/make_reference_fixtures.py [reference root]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from acoustics_b200.solver import read_obj  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"


def main():
    path = os.path.join(REF, "work", "meshes", "small_ball", "small_ball.obj")
    m = read_obj(path)
    np.savez_compressed(os.path.join(HERE, "small_ball_mesh.npz"), vertices=m.vertices, triangles=m.triangles,
                        source="work/meshes/small_ball/small_ball.obj")
    print(path, m.vertices.shape, m.triangles.shape)


if __name__ == "__main__":
    main()
