"""Kremer-Grest melt (WCA + FENE, Langevin, capped-LJ warm-up) on the GPU against the
oracle: the melt is built by tools.topology.polymer_melt, the run follows the
Kremer-Grest recipe (dt 0.01, gamma 0.5, T 1, pair force capped first: LennardJonesCapped
keeps FENE intact, where a cap on the total force lets bonds stretch past R0)."""
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from espressopp_b200.tools import topology
from simdriver import Sim, cell_grid, cuda_lib, oracle_lib

pytestmark = pytest.mark.gpu

RC = 2.0 ** (1.0 / 6.0)


SHIFT = 4.0 * ((1.0 / RC ** 2) ** 6 - (1.0 / RC ** 2) ** 3)  # 'auto'


def _kg(lib, prec, pos, bonds, L, seed=11):
    box = np.array([L, L, L])
    s = Sim(lib, box, 0.3, cell_grid(box, RC, 0.3), precision=prec, seed=seed)
    s.add(np.arange(1, len(pos) + 1), pos, np.zeros_like(pos))
    s.decompose()
    s.vl(RC)
    s.lj(0, 0, 1.0, 1.0, RC, SHIFT, caprad=0.9)
    s.bonds(bonds)
    s.fene(30.0, 0.0, 1.5)
    s.integrator(0.01)
    s.langevin(0.5, 1.0)
    return s


def test_kg_melt_warmup_and_run_match_oracle():
    pos, bonds, L = topology.polymer_melt(20, 50, 0.85, seed=3)
    sims = [_kg(oracle_lib(), _abi.PREC_FP64, pos, bonds, L),
            _kg(cuda_lib(), _abi.PREC_FP64, pos, bonds, L),
            _kg(cuda_lib(), _abi.PREC_MIXED, pos, bonds, L)]
    ids = np.arange(1, len(pos) + 1)
    for s in sims:
        s.run(100)
        s.lj(0, 0, 1.0, 1.0, RC, SHIFT)
        s.run(100)
    ref = sims[0].particles(ids)
    got = sims[1].particles(ids)
    assert np.max(np.abs(got[0] - ref[0])) < 1e-8
    assert np.array_equal(got[3], ref[3])
    # mixed precision: 2 tau of a dense Langevin melt amplifies the 1e-6 force differences
    # chaotically; positions (unfolded with their images) stay within a few 1e-3
    mx = sims[2].particles(ids)
    unf = lambda p: p[0] + p[3] * L
    assert np.max(np.abs(unf(mx) - unf(ref))) < 0.05
    for which in (_abi.IA_LJ, _abi.IA_FENE):
        eo = sims[0].energy(which)
        assert abs(sims[1].energy(which) - eo) < 1e-8 * abs(eo)
    # the melt is still relaxing its growth overlaps (the thermostat's time is 2 tau)
    v2, n = sims[1].kinetic()
    assert abs(v2 - sims[0].kinetic()[0]) < 1e-8 * v2 and 0.5 < v2 / (3 * n) < 5.0
    mx = np.zeros(1)
    _abi.call(sims[1].lib, "espp_bonds_max_sqr", sims[1].h, _abi.dptr(mx))
    assert math.sqrt(mx[0]) < 1.5


def _max_bond_sq(s):
    mx = np.zeros(1)
    _abi.call(s.lib, "espp_bonds_max_sqr", s.h, _abi.dptr(mx))
    return float(mx[0])


def _bond_sq_now(s, bonds, L, n):
    x = s.particles(np.arange(1, n + 1))[0]
    b = np.asarray(bonds) - 1
    d = x[b[:, 0]] - x[b[:, 1]]
    d -= L * np.round(d / L)
    return float(np.max(np.sum(d * d, axis=1)))


def test_longtime_max_bond_matches_oracle():
    """FixedPairList's long-time maximum bond length (FixedPairList.cpp:82-86, raised by
    every force pass in FixedPairListInteractionTemplate.hpp:116-150): 0 before the first
    force pass, the longest bond of that pass after it, never below the longest bond of
    the last pass after a run, 0 again after a reset; the GPU's value against the oracle's
    in both precisions.  An emptied list (FixedPairList::remove) raises it no more."""
    pos, bonds, L = topology.polymer_melt(20, 50, 0.85, seed=3)
    n = len(pos)
    sims = [_kg(oracle_lib(), _abi.PREC_FP64, pos, bonds, L),
            _kg(cuda_lib(), _abi.PREC_FP64, pos, bonds, L),
            _kg(cuda_lib(), _abi.PREC_MIXED, pos, bonds, L)]
    assert [_max_bond_sq(s) for s in sims] == [0.0, 0.0, 0.0]
    for s in sims:
        s.run(0)
    m = [_max_bond_sq(s) for s in sims]
    now = _bond_sq_now(sims[0], bonds, L, n)
    assert abs(m[0] - now) <= 1e-12 * now
    assert abs(m[1] - m[0]) <= 1e-12 * m[0]
    assert abs(m[2] - m[0]) <= 1e-5 * m[0]  # FP32 distances on box-wrapped coordinates
    for s in sims:
        _abi.call(s.lib, "espp_bonds_reset_max", s.h)
    assert [_max_bond_sq(s) for s in sims] == [0.0, 0.0, 0.0]
    for s in sims:
        s.run(30)
    m = [_max_bond_sq(s) for s in sims]
    for s, v in zip(sims, m):
        assert v >= _bond_sq_now(s, bonds, L, n) * (1 - 1e-5) and v < 1.5 ** 2
    assert abs(m[1] - m[0]) <= 1e-6 * m[0]
    assert abs(m[2] - m[0]) <= 1e-2 * m[0]
    for s in sims:
        _abi.call(s.lib, "espp_bonds_clear", s.h)
        _abi.call(s.lib, "espp_bonds_reset_max", s.h)
        s.run(5)
        assert _max_bond_sq(s) == 0.0 and s.energy(_abi.IA_FENE) == 0.0
    assert np.max(np.abs(sims[1].particles(np.arange(1, n + 1))[0]
                         - sims[0].particles(np.arange(1, n + 1))[0])) < 1e-6
