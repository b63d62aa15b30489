"""Coarse-graining workflow on the GPU at a small scale: fine-grained Kremer-Grest frames,
4:1 centre-of-mass mapping, Boltzmann-inverted bond table, force-matched pair table
(fallback), force-matching training of the learned potential, and a CG run."""
import math
import os

import numpy as np
import pytest

from espressopp_b200 import _abi, cg
from espressopp_b200._abi import call

pytestmark = pytest.mark.gpu


def test_cg_workflow_small(tmp_path):
    pos, frc, L, bonds = cg.fg_frames(24, 40, nframes=12, interval=10, warm_capped=200,
                                      warm=300, window=20)
    assert pos.shape == (12, 240, 3) and frc.shape == (12, 240, 3)
    # the mapped forces sum to zero (Newton's third law over the whole system)
    assert np.max(np.abs(frc.sum(axis=1))) < 1e-6 * np.abs(frc).sum() / 12
    lengths = cg.bond_lengths(pos, bonds)
    tab = cg.boltzmann_bond_table(lengths, path=str(tmp_path / "bond.tab"))
    assert os.path.exists(tmp_path / "bond.tab")
    zero = ([0.5, 1.0, 1.5, 2.0], [0.0] * 4, [0.0] * 4)
    bond_only = cg.CGSystem(pos[0], L, bonds, tab)
    fbond = np.array([bond_only.forces_at(p) for p in pos])
    target = frc - fbond
    ptab = cg.pair_fm_table(pos[:8], target[:8], L)
    pair_only = cg.CGSystem(pos[0], L, bonds, zero)
    pair_only.set_pair_table(ptab)
    # the least-squares pair table lowers the force error on the frames it was fitted to;
    # on the four held-out frames of this tiny melt it stays at the noise level
    err_fit = cg.fm_error(pair_only, pos[:8], target[:8])
    assert err_fit < 1.0
    err_table = cg.fm_error(pair_only, pos[8:], target[8:])
    assert err_table < 1.05
    resid = np.array([t - pair_only.forces_at(p) for p, t in zip(pos, target)])
    s = cg.CGSystem(pos[0], L, bonds, tab)
    triples = cg.angle_triples(bonds)
    assert len(triples) == 24 * (10 - 2)
    atab = cg.boltzmann_angle_table(cg.angles_of(pos, triples))
    assert np.all(np.isfinite(atab[1])) and atab[2][-1] == 0.0
    s.set_angle_table(triples, atab)
    s.set_pair_table(ptab)
    model = cg.MLPModel(seed=3)
    s.attach(model)
    shift, scale = cg.descriptor_norm(s, pos)
    model.set_norm(shift, scale)
    hist = cg.train_mlp(s, model, pos[:8], resid[:8], epochs=6, batch=2, lr=1e-3)
    assert hist[-1] < hist[0]
    err_mlp = cg.fm_error(s, pos[8:], target[8:], fbond[8:])
    assert math.isfinite(err_mlp)
    # CG dynamics with the learned potential and the bond table
    call(s.lib, "espp_set_particles", s.h, len(s.ids), _abi.i64ptr(s.ids),
         _abi.dptr(np.ascontiguousarray(cg.wrap(pos[-1], L)).reshape(-1)), None)
    call(s.lib, "espp_integrator_set", s.h, 0.01)
    s.thermostat(True)
    s.run(400)
    p, v, f, img = s.state(s.ids)
    T = np.sum(4.0 * v * v) / (3 * len(s.ids))
    assert np.all(np.isfinite(p)) and 0.6 < T < 1.5
    g = s.rdf(50)
    assert np.all(np.isfinite(g))
    model.close()
