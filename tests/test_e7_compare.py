"""The comparer restatement's distance rule (tests/e7_compare.py) on the CPU: planes and spheres in the collider
packing of problem.bin, points placed inside and outside."""
import numpy as np

from tests import e7_compare


def test_distances_to_planes_and_spheres():
    colliders = np.array([1, 0, 1, 0, -0.25, 0, 0, 0,     # plane y = -0.25
                          2, 0, 0, 0, 0.25, 0, 0, 0], float)  # sphere r = 0.25 at the origin
    x = np.array([0, 0.3, 0,        # above the sphere: 0.05 from it
                  0, 0.1, 0,        # inside the sphere: -0.15
                  0.9, -0.2, 0,     # above the floor, far from the sphere: 0.05 from the plane
                  0.9, -0.3, 0])    # below the floor: -0.05
    d = e7_compare.distances(colliders, x)
    assert np.allclose(d, [0.05, -0.15, 0.05, -0.05])
