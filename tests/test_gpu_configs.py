"""GPU parity against the FP64 oracle at the benchmark's own configurations.

* LJ fluid, 32,768 particles: 32^3 simple-cubic lattice at density 0.8442, uniform jitter
  +-0.05 sigma (PCG64 seed 1), Maxwell-Boltzmann velocities at T = 1 (seed 2, zero net
  momentum), cells 12^3, LJ eps = sigma = 1, rc = 2.5 shifted, skin 0.3, dt 0.005,
  Langevin gamma 1, T 1.  The sorted id-pair set equals the oracle's
  (VerletList.cpp:274-450), forces, energy, virial and its tensor agree, and a 200-step
  FP64 Langevin trajectory follows the oracle's with the same list builds and re-sorts.
* Large LJ fluid, 4,096,000 particles: 160^3 lattice, cells 60^3, NVE.  The pair set
  (compared through espp_vl_digest: 159 million pairs) equals the oracle's at the lattice
  and after a re-sort made inside the captured step loop, and the mixed-precision forces
  agree with the FP64 oracle.

Tolerances: FP64 forces 1e-12 relative RMS; mixed forces 1e-5 relative RMS and, per
particle, |dF_i| <= 5e-3 of the RMS force; energies and virials 1e-10 relative; FP64
trajectory 1e-9 absolute in positions and velocities.
"""
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import Sim, cell_grid, cuda_lib, lattice, mb_velocities, oracle_lib

pytestmark = pytest.mark.gpu

RC, SKIN, DT = 2.5, 0.3, 0.005
SHIFT = 4.0 * (RC ** -12 - RC ** -6)
MAX_REL_PER_PARTICLE = 5e-3


def _system(lib, prec, ids, pos, vel, box, langevin, seed=2024):
    s = Sim(lib, box, SKIN, cell_grid(box, RC, SKIN), precision=prec, seed=seed)
    s.add(ids, pos, vel)
    s.decompose()
    s.vl(RC)
    s.lj(0, 0, 1.0, 1.0, RC, SHIFT)
    s.integrator(DT)
    if langevin:
        s.langevin(1.0, 1.0)
    return s


def _force_errors(f, fref):
    df = f - fref
    rms = math.sqrt(np.sum(df * df) / np.sum(fref * fref))
    per = float(np.max(np.linalg.norm(df, axis=1)) /
                math.sqrt(np.mean(np.sum(fref * fref, axis=1))))
    return rms, per


@pytest.fixture(scope="module")
def config1():
    pos, box = lattice(32, 0.8442, 0.05, 1)
    vel = mb_velocities(len(pos), 1.0, 2)
    ids = np.arange(len(pos), dtype=np.int64)
    assert cell_grid(box, RC, SKIN) == [12, 12, 12]
    o = _system(oracle_lib(), _abi.PREC_FP64, ids, pos, vel, box, langevin=True)
    o.run(0)
    return ids, pos, vel, box, o


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_config1_pairs_forces_observables(config1, prec):
    ids, pos, vel, box, o = config1
    g = _system(cuda_lib(), prec, ids, pos, vel, box, langevin=True)
    po, pg = o.pairs(), g.pairs()
    assert len(po) == g.vl_size() and np.array_equal(po, pg)
    assert g.digest() == o.digest()
    g.run(0)
    fo = o.particles(ids)[2]
    fg = g.particles(ids)[2]
    rms, per = _force_errors(fg, fo)
    if prec == _abi.PREC_FP64:
        assert rms < 1e-12
    else:
        assert rms < 1e-5 and per < MAX_REL_PER_PARTICLE
    eo, wo = o.energy(_abi.IA_LJ), o.virial(_abi.IA_LJ)
    assert abs(g.energy(_abi.IA_LJ) - eo) < 1e-10 * abs(eo)
    assert abs(g.virial(_abi.IA_LJ) - wo) < 1e-10 * abs(wo)
    to, tg = o.virial_tensor(_abi.IA_LJ), g.virial_tensor(_abi.IA_LJ)
    assert np.all(np.abs(tg - to) <= 1e-10 * np.max(np.abs(to)))


def test_config1_fp64_langevin_trajectory_200_steps():
    pos, box = lattice(32, 0.8442, 0.05, 1)
    vel = mb_velocities(len(pos), 1.0, 2)
    ids = np.arange(len(pos), dtype=np.int64)
    sims = [_system(lib, _abi.PREC_FP64, ids, pos, vel, box, langevin=True)
            for lib in (oracle_lib(), cuda_lib())]
    for s in sims:
        s.run(200)
    (xo, vo, _, io), (xg, vg, _, ig) = (s.particles(ids) for s in sims)
    assert np.max(np.abs(xg - xo)) < 1e-9 and np.max(np.abs(vg - vo)) < 1e-9
    assert np.array_equal(ig, io)
    assert sims[1].builds() == sims[0].builds() and sims[1].builds() > 1
    assert sims[1].num_resorts() == sims[0].num_resorts()
    assert np.array_equal(sims[0].pairs(), sims[1].pairs())


def _oracle_at(ids, pos, box):
    o = _system(oracle_lib(), _abi.PREC_FP64, ids, pos, None, box, langevin=False)
    o.run(0)
    return o


def test_config3_pair_set_and_mixed_forces_4M():
    """4,096,000 particles: the in-graph list (int32 list offsets, grown capacity, 60^3
    cells, 32-bit coordinate wrap at L = 169.3) against the oracle's."""
    pos, box = lattice(160, 0.8442, 0.05, 1)
    vel = mb_velocities(len(pos), 1.0, 2)
    ids = np.arange(len(pos), dtype=np.int64)
    assert cell_grid(box, RC, SKIN) == [60, 60, 60]
    g = _system(cuda_lib(), _abi.PREC_MIXED, ids, pos, vel, box, langevin=False)
    g.run(0)
    o = _oracle_at(ids, pos, box)
    assert g.digest() == o.digest()
    rms, per = _force_errors(g.particles(ids)[2], o.particles(ids)[2])
    assert rms < 1e-5 and per < MAX_REL_PER_PARTICLE
    del o
    # step until a re-sort happens inside the captured loop (num_resorts counts the
    # re-sorts of the last run): the list then in use was built at the positions the
    # run ends on (integrate2 moves no particle)
    for _ in range(40):
        g.run(1)
        if g.num_resorts() > 0:
            break
    assert g.num_resorts() > 0
    x, _, f, _ = g.particles(ids)
    o = _oracle_at(ids, x, box)
    assert g.digest() == o.digest()
    rms, per = _force_errors(f, o.particles(ids)[2])
    assert rms < 1e-5 and per < MAX_REL_PER_PARTICLE
