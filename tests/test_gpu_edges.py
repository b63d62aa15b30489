"""Edge cases on the GPU against the FP64 oracle: an empty system, one particle, particles
on and just outside the box faces, and a pair exactly at the Verlet cutoff (the
reference's inclusion test is !(d^2 > cutsq), VerletList.cpp:434-450)."""
import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import Sim, cuda_lib, oracle_lib

pytestmark = pytest.mark.gpu

BOX = [12.0, 12.0, 12.0]
GRID = [4, 4, 4]  # cells of 3.0 >= rc + skin = 2.8


def _setup(lib, ids, pos, vel=None, prec=_abi.PREC_FP64):
    s = Sim(lib, BOX, 0.3, GRID, precision=prec, seed=9)
    if len(ids):
        s.add(ids, pos, vel)
    s.decompose()
    s.vl(2.5)
    s.lj(0, 0, 1.0, 1.0, 2.5, 0.0)
    s.integrator(0.005)
    return s


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_empty_system_runs(prec):
    for lib in (oracle_lib(), cuda_lib()):
        s = _setup(lib, np.zeros(0, np.int64), np.zeros((0, 3)), prec=prec)
        s.run(5)
        assert s.energy(_abi.IA_LJ) == 0.0
        assert s.vl_size() == 0 and len(s.pairs()) == 0
        assert s.kinetic() == (0.0, 0)


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_single_particle_moves_ballistically(prec):
    ids = np.array([5])
    pos = np.array([[11.9, 0.05, 6.0]])
    vel = np.array([[1.5, -0.7, 0.25]])
    out = []
    for lib in (oracle_lib(), cuda_lib()):
        s = _setup(lib, ids, pos, vel, prec=prec)
        s.run(40)
        out.append(s.particles(ids))
    (po, vo, fo, io), (pg, vg, fg, ig) = out
    assert np.array_equal(pg, po) and np.array_equal(vg, vo) and np.array_equal(ig, io)
    assert np.all(fg == 0.0)
    # crossed the +x and -y faces: folded positions and image counts
    assert ig[0, 0] == 1 and ig[0, 1] == -1


def test_particles_on_and_outside_the_faces():
    """Positions at 0, at L, a hair below 0 and a hair below L fold as the reference
    folds them; pairs across the faces are found, and forces agree."""
    L = BOX[0]
    pos = np.array([[0.0, 6.0, 6.0], [L, 6.5, 6.0], [-1e-12, 5.0, 6.0],
                    [L - 1e-12, 5.5, 7.0], [11.2, 11.99999999, 0.0], [0.6, 0.0, 11.8],
                    [6.0, 6.0, 6.0]])
    ids = np.arange(1, len(pos) + 1)
    o = _setup(oracle_lib(), ids, pos)
    g = _setup(cuda_lib(), ids, pos)
    assert np.array_equal(o.pairs(), g.pairs())
    po, pg = o.particles(ids), g.particles(ids)
    assert np.array_equal(pg[0], po[0]) and np.array_equal(pg[3], po[3])
    for s in (o, g):
        s.run(0)
    assert np.allclose(g.particles(ids)[2], o.particles(ids)[2], rtol=1e-12, atol=1e-12)


def test_pair_exactly_at_the_verlet_cutoff():
    """|d|^2 == (rc + skin)^2 in FP64 is inside (!(d2 > cutsq)); one ulp further is out."""
    cut = 2.5 + 0.3
    x0 = 4.0
    inside = x0 + cut          # d = cut exactly: d*d == cut*cut
    outside = np.nextafter(inside, np.inf)
    assert (inside - x0) ** 2 == cut * cut and (outside - x0) ** 2 > cut * cut
    pos = np.array([[x0, 6.0, 6.0], [inside, 6.0, 6.0], [x0, 2.0, 2.0], [outside, 2.0, 2.0]])
    ids = np.array([1, 2, 3, 4])
    o = _setup(oracle_lib(), ids, pos)
    g = _setup(cuda_lib(), ids, pos)
    po, pg = o.pairs(), g.pairs()
    assert np.array_equal(po, pg)
    assert [1, 2] in po.tolist() and [3, 4] not in po.tolist()
