"""Host-side pieces of the coarse-graining workflow (numpy only): angle triples of the
chains, bending angles, and the Boltzmann-inverted angle table."""
import math

import numpy as np

from espressopp_b200 import cg


def test_angle_triples_follow_the_chains():
    bonds = np.array([[k, k + 1] for c in range(3) for k in range(c * 10 + 1, c * 10 + 10)])
    t = cg.angle_triples(bonds)
    assert t.shape == (3 * 8, 3)
    assert t[0].tolist() == [1, 2, 3] and t[7].tolist() == [8, 9, 10]
    assert [10, 11, 12] not in t.tolist()  # no triple across chains


def test_angles_of_frames():
    p = np.array([[[0.0, 0, 0], [1.0, 0, 0], [1.0, 1.0, 0], [2.0, 1.0, 0]]])
    t = np.array([[1, 2, 3], [2, 3, 4]])
    assert np.allclose(cg.angles_of(p, t), [math.pi / 2, math.pi / 2])


def test_boltzmann_angle_table_recovers_a_known_potential():
    rng = np.random.default_rng(0)
    x = rng.uniform(0.0, math.pi, 2_000_000)
    w = np.sin(x) * np.exp(-2.0 * (np.cos(x) + 0.6) ** 2)  # P(theta) for U = 2 (cos + 0.6)^2
    th = x[rng.uniform(0.0, 1.0, x.size) < w / w.max()]
    T, E, F = cg.boltzmann_angle_table(th)
    U = 2.0 * (np.cos(T) + 0.6) ** 2
    sel = T > 1.2
    dev = (E - E[sel].min())[sel] - (U - U[sel].min())[sel]
    assert np.max(np.abs(dev)) < 0.08
    assert F[-1] == 0.0 and np.all(np.isfinite(E)) and np.all(np.isfinite(F))
    # the force f = -dE/dtheta vanishes towards pi, so f / sin(theta) stays finite
    assert abs(F[-2]) < 0.2
