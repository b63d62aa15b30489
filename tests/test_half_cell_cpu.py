"""halfCellInt on the CPU oracle (DomainDecomposition.cpp:325-357, tools/decomp.py:322):
the fine cell grid with a (2h+1)^3 neighbour stencil and an h-cell ghost frame.

With cells at least cutoff/h wide every pair within the cutoff lies in the stencil, so the
Verlet list equals the brute-force minimum-image pair set; an h = 2 run follows the h = 1
run of the same system.  The ABI rejects bad values, and the Python mirror passes
storage.DomainDecomposition(..., halfCellInt) through.
"""
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import Sim, cell_grid, lattice, mb_velocities, oracle_lib

RC, SKIN = 2.5, 0.3


def _brute_pairs(ids, pos, box, cut):
    d = pos[:, None, :] - pos[None, :, :]
    d -= box * np.round(d / box)
    r2 = np.sum(d * d, axis=2)
    i, j = np.nonzero(np.triu(r2 <= cut * cut, 1))
    p = np.stack([ids[i], ids[j]], 1)
    p = np.sort(p, axis=1)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def _fluid(h, pos, vel, box, langevin=False):
    ids = np.arange(len(pos), dtype=np.int64)
    s = Sim(oracle_lib(), box, SKIN, cell_grid(box, RC, SKIN, h), seed=4, half_cell_int=h)
    s.add(ids, pos, vel)
    s.decompose()
    s.vl(RC)
    s.lj(0, 0, 1.0, 1.0, RC, 4.0 * (RC ** -12 - RC ** -6))
    s.integrator(0.005)
    if langevin:
        s.langevin(1.0, 1.0)
    return s


@pytest.mark.parametrize("h", [1, 2, 3])
def test_pairs_equal_brute_force(h):
    rng = np.random.Generator(np.random.PCG64(7))
    box = np.array([17.0, 15.5, 16.3])
    pos = rng.uniform(0, 1, size=(3000, 3)) * box
    ids = np.arange(len(pos), dtype=np.int64)
    s = _fluid(h, pos, None, box)
    assert all(c >= 2 * h + 1 for c in cell_grid(box, RC, SKIN, h))
    assert np.array_equal(s.pairs(), _brute_pairs(ids, pos, box, RC + SKIN))


def test_half_cell_run_follows_full_cells():
    pos, box = lattice(10, 0.8442, 0.05, 3)
    vel = mb_velocities(len(pos), 1.0, 4)
    ids = np.arange(len(pos), dtype=np.int64)
    runs = [_fluid(h, pos, vel, box, langevin=True) for h in (1, 2)]
    for s in runs:
        s.run(60)
    (x1, v1, _, i1), (x2, v2, _, i2) = (s.particles(ids) for s in runs)
    assert np.max(np.abs(x2 - x1)) < 1e-9 and np.max(np.abs(v2 - v1)) < 1e-9
    assert np.array_equal(i1, i2)
    assert runs[0].builds() == runs[1].builds() > 1
    assert np.array_equal(runs[0].pairs(), runs[1].pairs())
    e1, e2 = runs[0].energy(_abi.IA_LJ), runs[1].energy(_abi.IA_LJ)
    assert abs(e1 - e2) < 1e-9 * abs(e1)


def test_half_cell_argument_checks():
    lib = oracle_lib()
    box = np.array([20.0, 20.0, 20.0])
    s = Sim(lib, box, SKIN, [7, 7, 7])
    for bad in (0, 5):
        with pytest.raises(RuntimeError):
            _abi.call(lib, "espp_set_half_cell_int", s.h, bad)
    with pytest.raises(RuntimeError):  # 7 cells < 2 * 4 + 1
        _abi.call(lib, "espp_set_half_cell_int", s.h, 4)
    _abi.call(lib, "espp_set_half_cell_int", s.h, 3)
    s.add(np.arange(2), np.array([[1.0, 1.0, 1.0], [2.0, 2.0, 2.0]]))
    with pytest.raises(RuntimeError):  # particles present
        _abi.call(lib, "espp_set_half_cell_int", s.h, 2)


def test_mirror_half_cell_int():
    import espressopp_b200 as espressopp
    from espressopp_b200 import _lib
    saved = _lib._lib
    _lib._lib = oracle_lib()
    try:
        out = []
        for h in (1, 2):
            x, y, z, Lx, Ly, Lz = espressopp.tools.lattice.createCubic(
                1000, 0.8442, perfect=False, RNG=espressopp.esutil.RNG(5))
            system = espressopp.System()
            system.rng = espressopp.esutil.RNG(6)
            system.bc = espressopp.bc.OrthorhombicBC(system.rng, (Lx, Ly, Lz))
            system.skin = SKIN
            cg = espressopp.tools.decomp.cellGrid((Lx, Ly, Lz), (1, 1, 1), RC, SKIN, h)
            system.storage = espressopp.storage.DomainDecomposition(system, (1, 1, 1), cg,
                                                                    halfCellInt=h)
            system.storage.addParticles([[k, espressopp.Real3D(x[k], y[k], z[k])]
                                         for k in range(len(x))], "id", "pos")
            system.storage.decompose()
            vl = espressopp.VerletList(system, cutoff=RC)
            lj = espressopp.interaction.VerletListLennardJones(vl)
            lj.setPotential(0, 0, espressopp.interaction.LennardJones(1.0, 1.0, RC, "auto"))
            system.addInteraction(lj)
            out.append((lj.computeEnergy(), vl.totalSize()))
        assert out[0][1] == out[1][1]
        assert math.isclose(out[0][0], out[1][0], rel_tol=1e-12)
    finally:
        _lib._lib = saved
