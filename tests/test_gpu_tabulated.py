"""GPU parity of interaction::Tabulated (VerletListTabulated, FixedPairListTabulated)
against the oracle, and the reference's tabulated step-0 energies
(testsuite/tabulated/result.dat)."""
import math

import numpy as np
import pytest

from espressopp_b200 import _abi, interaction
from simdriver import (Sim, cell_grid, cuda_lib, lattice, load_polymer40k, mb_velocities,
                       oracle_lib, polymer_tab_tables, read_tab, write_tab_file)

pytestmark = pytest.mark.gpu


def _rel_rms(a, b):
    return math.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2))


def _tab_pair(s, t1, t2, itype, tab, rc, shift=0.0):
    r, e, f = tab
    _abi.call(s.lib, "espp_tab_pair_set", s.h, t1, t2, itype, len(r), _abi.dptr(r),
              _abi.dptr(e), _abi.dptr(f), rc, shift)


def _tab_bond(s, itype, tab, rc=math.inf):
    r, e, f = tab
    _abi.call(s.lib, "espp_tab_bond_set", s.h, itype, len(r), _abi.dptr(r), _abi.dptr(e),
              _abi.dptr(f), rc, 0.0)


def _polymer(lib, prec, tabs, itype=2):
    pos, bonds, box, gold = load_polymer40k()
    s = Sim(lib, box, 0.3, cell_grid(box, 1.12, 0.3), precision=prec, seed=5)
    s.add(np.arange(1, len(pos) + 1), pos)
    s.decompose()
    s.vl(1.42)
    s.bonds(bonds)
    _tab_pair(s, 0, 0, itype, tabs[0], 1.12)
    _tab_bond(s, itype, tabs[1])
    return s, gold


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_tabulated_polymer_melt_golden_step0(tmp_path, prec):
    tl, tf, _, _ = polymer_tab_tables(tmp_path, cuda_lib())
    s, gold = _polymer(cuda_lib(), prec, (tl, tf))
    g = gold["tabulated"]
    assert round(s.energy(_abi.IA_TAB_PAIR), 3) == g["epair"]
    assert round(s.energy(_abi.IA_TAB_BOND), 3) == g["ebond"]


@pytest.mark.parametrize("itype", [1, 2, 3])
def test_tabulated_forces_and_observables_match_oracle(tmp_path, itype):
    tl, tf, _, _ = polymer_tab_tables(tmp_path, oracle_lib())
    o, _ = _polymer(oracle_lib(), _abi.PREC_FP64, (tl, tf), itype)
    g64, _ = _polymer(cuda_lib(), _abi.PREC_FP64, (tl, tf), itype)
    gmx, _ = _polymer(cuda_lib(), _abi.PREC_MIXED, (tl, tf), itype)
    ids = np.arange(1, 40001)
    for s in (o, g64, gmx):
        s.integrator(0.01)
        s.run(0)
    fo = o.particles(ids)[2]
    assert _rel_rms(g64.particles(ids)[2], fo) < 1e-12
    assert _rel_rms(gmx.particles(ids)[2], fo) < 1e-9
    # the bond list's long-time maximum, raised by the tabulated bond pass on FP64
    # distances in both precisions
    mx = np.zeros(3)
    for k, s in enumerate((o, g64, gmx)):
        _abi.call(s.lib, "espp_bonds_max_sqr", s.h, _abi.dptr(mx[k:]))
    assert mx[0] > 0 and np.all(np.abs(mx[1:] - mx[0]) <= 1e-14 * mx[0])
    for which in (_abi.IA_TAB_PAIR, _abi.IA_TAB_BOND):
        eo, wo = o.energy(which), o.virial(which)
        for g in (g64, gmx):
            assert abs(g.energy(which) - eo) < 1e-10 * abs(eo)
            assert abs(g.virial(which) - wo) < 1e-10 * abs(wo)
        assert np.allclose(g64.virial_tensor(which), o.virial_tensor(which), rtol=1e-9,
                           atol=1e-9)


def test_tabulated_langevin_run_matches_oracle(tmp_path):
    tl, tf, _, _ = polymer_tab_tables(tmp_path, oracle_lib())
    sims = [_polymer(oracle_lib(), _abi.PREC_FP64, (tl, tf), 3)[0],
            _polymer(cuda_lib(), _abi.PREC_FP64, (tl, tf), 3)[0],
            _polymer(cuda_lib(), _abi.PREC_MIXED, (tl, tf), 3)[0]]
    ids = np.arange(1, 40001)
    for s in sims:
        s.integrator(0.002)
        s.langevin(1.0, 1.0)
        s.run(30)
    ref = sims[0].particles(ids)
    for s, tol in ((sims[1], 1e-9), (sims[2], 1e-5)):
        got = s.particles(ids)
        assert np.max(np.abs(got[0] - ref[0])) < tol
        assert _rel_rms(got[1], ref[1]) < tol
    assert sims[1].num_resorts() == sims[0].num_resorts()


def test_lj_and_tabulated_on_one_verlet_list(tmp_path):
    """Two types: (0,0) Lennard-Jones, (0,1) and (1,1) tabulated; energies per interaction
    and the forces of both interactions together match the oracle."""
    pos, box = lattice(14, 0.8442, 0.05, seed=3)
    n = len(pos)
    types = (np.arange(n) % 3 == 0).astype(np.int32)
    vel = mb_velocities(n, 1.0, seed=4)
    soft = interaction.LennardJones(0.7, 1.1, cutoff=2.5)
    path = str(tmp_path / "soft.tab")
    write_tab_file(soft, path, N=400, low=0.6, high=2.6)
    tab = read_tab(oracle_lib(), path)
    sims = []
    for lib, prec in ((oracle_lib(), _abi.PREC_FP64), (cuda_lib(), _abi.PREC_FP64),
                      (cuda_lib(), _abi.PREC_MIXED)):
        s = Sim(lib, box, 0.3, cell_grid(box, 2.5, 0.3), precision=prec, seed=9)
        s.add(np.arange(n), pos, vel, types=types)
        s.decompose()
        s.vl(2.5)
        s.lj(0, 0, 1.0, 1.0, 2.5, 0.0)
        _tab_pair(s, 0, 1, 3, tab, 2.5, shift=0.01)
        _tab_pair(s, 1, 1, 1, tab, 2.2)
        s.integrator(0.004)
        s.run(0)
        sims.append(s)
    fo = sims[0].particles(np.arange(n))[2]
    assert _rel_rms(sims[1].particles(np.arange(n))[2], fo) < 1e-12
    assert _rel_rms(sims[2].particles(np.arange(n))[2], fo) < 1e-5
    for which in (_abi.IA_LJ, _abi.IA_TAB_PAIR):
        eo = sims[0].energy(which)
        for s in sims[1:]:
            assert abs(s.energy(which) - eo) < 1e-10 * abs(eo)
    for s in sims:
        s.run(25)
    ref = sims[0].particles(np.arange(n))
    got = sims[1].particles(np.arange(n))
    assert np.max(np.abs(got[0] - ref[0])) < 1e-9
