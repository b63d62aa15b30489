"""Verlet-list parity in geometries that stress the build's grouping (32 consecutive
particles of one row of cells, split where the row changes or the group would span too
many x-cells) and its x-cell range with periodic wrap, against the FP64 oracle
(VerletList.cpp:274-450):

* a dilute gas (0.4 particles per cell): groups span many cells and split by span;
* the smallest grid the run form takes in x (3 cells) with long y and z;
* a slab: particles only in a third of the box, so most rows are empty;
* cells just above the cutoff (0.2 %: the run form; 0.05 %: the per-cell form);
and a grid of 2 cells in one dimension, which the GPU storage refuses.
Each compares the sorted id-pair sets, the pair digests and the mixed-precision forces.
"""
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import Sim, cuda_lib, oracle_lib

pytestmark = pytest.mark.gpu

RC, SKIN = 2.5, 0.3
SHIFT = 4.0 * (RC ** -12 - RC ** -6)


def _both(pos, box, grid, prec=_abi.PREC_MIXED):
    ids = np.arange(len(pos), dtype=np.int64)
    out = []
    for lib, p in ((oracle_lib(), _abi.PREC_FP64), (cuda_lib(), prec)):
        s = Sim(lib, box, SKIN, grid, precision=p, seed=3)
        s.add(ids, pos)
        s.decompose()
        s.vl(RC)
        s.lj(0, 0, 1.0, 1.0, RC, SHIFT)
        s.integrator(0.001)
        s.run(0)
        out.append(s)
    o, g = out
    assert g.vl_size() == o.vl_size()
    assert np.array_equal(g.pairs(), o.pairs())
    assert g.digest() == o.digest()
    fo, fg = o.particles(ids)[2], g.particles(ids)[2]
    if np.sum(fo * fo) > 0:
        assert math.sqrt(np.sum((fg - fo) ** 2) / np.sum(fo * fo)) < 1e-5
    return o, g


def _jittered(rng, box, a=1.15, jitter=0.15):
    """A simple-cubic lattice of spacing about a filling the box, jittered uniformly."""
    n = [max(1, int(b / a)) for b in box]
    g = [(np.arange(k) + 0.5) * (b / k) for k, b in zip(n, box)]
    p = np.stack(np.meshgrid(*g, indexing="ij"), -1).reshape(-1, 3)
    return p + rng.uniform(-jitter, jitter, size=p.shape)


def _spread(rng, n, box, dmin=0.9):
    """n points in the box at least dmin apart (dart throwing on a fine grid)."""
    pts = []
    tries = 0
    while len(pts) < n and tries < 200 * n:
        tries += 1
        p = rng.uniform(0, 1, 3) * box
        if pts:
            d = np.asarray(pts) - p
            d -= box * np.round(d / box)
            if np.min(np.sum(d * d, axis=1)) < dmin * dmin:
                continue
        pts.append(p)
    return np.asarray(pts)


def test_dilute_gas():
    rng = np.random.Generator(np.random.PCG64(21))
    box = np.array([60.0, 57.0, 55.0])
    pos = _spread(rng, 3000, box)
    grid = [int(b / (RC + SKIN)) for b in box]
    assert 3000 / np.prod(grid) < 0.5
    o, g = _both(pos, box, grid)
    assert g.vl_size() > 0


def test_three_cells_in_x():
    rng = np.random.Generator(np.random.PCG64(22))
    box = np.array([3 * 2.85, 30.0, 28.0])
    pos = _spread(rng, 1500, box)
    grid = [3, int(30.0 / 2.8), int(28.0 / 2.8)]
    _both(pos, box, grid)


def test_slab_with_empty_rows():
    rng = np.random.Generator(np.random.PCG64(23))
    box = np.array([34.0, 34.0, 34.0])
    pos = _spread(rng, 4000, np.array([34.0, 34.0, 11.0]))
    grid = [int(b / (RC + SKIN)) for b in box]
    _both(pos, box, grid)


@pytest.mark.parametrize("edge", [2.8 * 1.002, 2.8 * 1.0005])
def test_cells_just_above_the_cutoff(edge):
    """Edges 0.2 % above the cutoff take the run form, 0.05 % the per-cell form."""
    rng = np.random.Generator(np.random.PCG64(24))
    grid = [10, 9, 11]
    box = np.array(grid, float) * edge
    _both(_jittered(rng, box), box, grid)


def test_two_cells_in_one_dimension_is_refused():
    """The GPU storage wants at least 3 cells per dimension (every neighbour cell of the
    27-cell stencil distinct); a smaller grid is refused with the reason, not built."""
    with pytest.raises(RuntimeError, match="at least 3 cells per dimension"):
        Sim(cuda_lib(), np.array([5.8, 25.0, 25.0]), SKIN, [2, 8, 8])
