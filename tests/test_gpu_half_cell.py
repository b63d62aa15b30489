"""halfCellInt on the GPU against the FP64 oracle (DomainDecomposition.cpp:325-357): the
fine cell grid and its (2h+1)^3 stencil give the oracle's pair set, bit-exact, for lists
built right after binning and for a rebuild on the cells of an earlier re-sort (where
particles may have left their cells and only the stencil cells count), with and without
exclusions; forces, energies and an FP64 Langevin trajectory follow the oracle's.
"""
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import (Sim, cell_grid, cuda_lib, lattice, load_polymer40k, mb_velocities,
                       oracle_lib)

pytestmark = pytest.mark.gpu

RC, SKIN = 2.5, 0.3
SHIFT = 4.0 * (RC ** -12 - RC ** -6)


def _fluid(lib, prec, h, ids, pos, vel, box, langevin=False):
    s = Sim(lib, box, SKIN, cell_grid(box, RC, SKIN, h), precision=prec, seed=8,
            half_cell_int=h)
    s.add(ids, pos, vel)
    s.decompose()
    s.vl(RC)
    s.lj(0, 0, 1.0, 1.0, RC, SHIFT)
    s.integrator(0.005)
    if langevin:
        s.langevin(1.0, 1.0)
    return s


def _rel_rms(a, b):
    return math.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2))


@pytest.mark.parametrize("h", [2, 3])
@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_fluid_pairs_forces(h, prec):
    pos, box = lattice(24, 0.8442, 0.05, 3)
    vel = mb_velocities(len(pos), 1.0, 4)
    ids = np.arange(len(pos), dtype=np.int64)
    o = _fluid(oracle_lib(), _abi.PREC_FP64, h, ids, pos, vel, box)
    g = _fluid(cuda_lib(), prec, h, ids, pos, vel, box)
    assert np.array_equal(g.pairs(), o.pairs())
    assert g.digest() == o.digest()
    o.run(0)
    g.run(0)
    tol = 1e-12 if prec == _abi.PREC_FP64 else 1e-5
    assert _rel_rms(g.particles(ids)[2], o.particles(ids)[2]) < tol
    eo = o.energy(_abi.IA_LJ)
    assert abs(g.energy(_abi.IA_LJ) - eo) < 1e-10 * abs(eo)


def test_fp64_langevin_trajectory_and_stale_rebuild():
    pos, box = lattice(16, 0.8442, 0.05, 5)
    vel = mb_velocities(len(pos), 1.0, 6)
    ids = np.arange(len(pos), dtype=np.int64)
    sims = [_fluid(lib, _abi.PREC_FP64, 2, ids, pos, vel, box, langevin=True)
            for lib in (oracle_lib(), cuda_lib())]
    for s in sims:
        s.run(120)
    (xo, vo, _, io), (xg, vg, _, ig) = (s.particles(ids) for s in sims)
    assert np.max(np.abs(xg - xo)) < 1e-9 and np.max(np.abs(vg - vo)) < 1e-9
    assert np.array_equal(ig, io)
    assert sims[1].builds() == sims[0].builds() > 1
    assert sims[1].num_resorts() == sims[0].num_resorts()
    # a few more steps without a re-sort, then a rebuild on the cells of the last re-sort
    for s in sims:
        s.run(2)
        s.vl_rebuild()
    assert np.array_equal(sims[0].pairs(), sims[1].pairs())


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_melt_fene_exclusions(prec):
    pos, bonds, box, _ = load_polymer40k()
    ids = np.arange(1, len(pos) + 1, dtype=np.int64)
    sims = []
    for lib, p in ((oracle_lib(), _abi.PREC_FP64), (cuda_lib(), prec)):
        s = Sim(lib, box, 0.3, cell_grid(box, 1.12, 0.3, 2), precision=p, half_cell_int=2)
        s.add(ids, pos)
        s.decompose()
        s.vl(1.42, excl=bonds)
        s.lj(0, 0, 1.0, 1.0, 1.12, 0.0)
        s.bonds(bonds)
        s.fene(30.0, 0.0, 1.5)
        s.integrator(0.005)
        s.run(0)
        sims.append(s)
    assert np.array_equal(sims[1].pairs(), sims[0].pairs())
    ex = set(map(tuple, np.sort(bonds, axis=1)))
    assert not ex & set(map(tuple, sims[1].pairs()))
    tol = 1e-12 if prec == _abi.PREC_FP64 else 1e-5
    assert _rel_rms(sims[1].particles(ids)[2], sims[0].particles(ids)[2]) < tol
    for w in (_abi.IA_LJ, _abi.IA_FENE):
        e0 = sims[0].energy(w)
        assert abs(sims[1].energy(w) - e0) < 1e-9 * abs(e0)


def test_half_cell_argument_checks():
    s = Sim(cuda_lib(), np.array([20.0, 20.0, 20.0]), SKIN, [7, 7, 7])
    for bad in (0, 5, 4):
        with pytest.raises(RuntimeError):
            _abi.call(s.lib, "espp_set_half_cell_int", s.h, bad)
    _abi.call(s.lib, "espp_set_half_cell_int", s.h, 3)
    s.add(np.arange(2), np.array([[1.0, 1.0, 1.0], [2.0, 2.0, 2.0]]))
    with pytest.raises(RuntimeError):
        _abi.call(s.lib, "espp_set_half_cell_int", s.h, 2)
