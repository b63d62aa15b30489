"""The FP64 oracle pinned to the reference's own golden values (CPU only).

Sources of the expected numbers (all inside espressopp/espressopp):
* testsuite/interaction_potentials/unittest/TestFENE.cpp:31-68 (FENE energies, force)
* testsuite/interaction_potentials/unittest/TestLennardJones.cpp:30-50 and
  testLennardJones.py (LJ minimum, zero crossing, cutoff)
* testsuite/interaction_potentials/unittest/testFENE.py (FENE at r0)
* testsuite/tabulated/result.dat:15-17 (step-0 energies and pressure of the 40 000-bead
  polymer melt), via tests/golden/polymer_melt_40k.*
* testsuite/unittest/PTestVerletList.cpp (Verlet list size == brute-force count)
* Random123 known-answer vectors for Philox4x32-10 (kat_vectors).
"""
import ctypes
import itertools
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import (Sim, cell_grid, cosine_angle_table, lattice, load_lj2048, load_polymer40k,
                       mb_velocities, msd_chain_reference, msd_reference, oracle_lib,
                       pair_digest)


def _lj(eps, sig, rc, shift, d, caprad=0.0):
    lib = oracle_lib()
    e = ctypes.c_double()
    f = (ctypes.c_double * 3)()
    dd = (ctypes.c_double * 3)(*d)
    lib.espp_oracle_lj_eval(eps, sig, rc, shift, caprad, dd, ctypes.byref(e), f)
    return e.value, list(f)


def _fene(K, r0, rmax, d, rc=math.inf, shift=0.0):
    lib = oracle_lib()
    e = ctypes.c_double()
    f = (ctypes.c_double * 3)()
    dd = (ctypes.c_double * 3)(*d)
    lib.espp_oracle_fene_eval(K, r0, rmax, rc, shift, dd, ctypes.byref(e), f)
    return e.value, list(f)


def test_philox_known_answers():
    lib = oracle_lib()
    cases = [
        ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
        ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
        ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
         [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
    ]
    for c, k, want in cases:
        C = (ctypes.c_uint32 * 4)(*c)
        K = (ctypes.c_uint32 * 2)(*k)
        O = (ctypes.c_uint32 * 4)()
        lib.espp_oracle_philox(C, K, O)
        assert list(O) == want


def test_fene_golden():
    # TestFENE.cpp: BOOST_CHECK_CLOSE(..., 0.01) is a 0.01 % tolerance
    for r, want in ((0.97, 18.279), (0.80, 11.296), (1.40, 69.147)):
        e, _ = _fene(30.0, 0.0, 1.5, (r, 0.0, 0.0))
        assert e == pytest.approx(want, rel=1e-4)
    _, f = _fene(30.0, 0.0, 1.5, (0.9, 0.1, 0.1))
    assert f == pytest.approx([-42.782, -4.7535, -4.7535], rel=1e-4)
    # testFENE.py: K=1, r0=1, rMax=0.5: E(1) = 0, F(1) = 0
    e, f = _fene(1.0, 1.0, 0.5, (1.0, 0.0, 0.0))
    assert e == 0.0 and f == [0.0, 0.0, 0.0]


def test_lj_golden():
    e, f = _lj(1.0, 1.0, math.inf, 0.0, (2 ** (1 / 6), 0, 0))
    assert e == pytest.approx(-1.0, rel=1e-4)
    assert abs(f[0]) < 1e-12
    assert abs(_lj(1.0, 1.0, math.inf, 0.0, (2.5, 0, 0))[0]) < 5.0
    assert abs(_lj(1.0, 1.0, math.inf, 0.0, (10.0, 0, 0))[0]) < 1.0
    # cutoff 2: small before, zero after (auto shift = E_raw(rc))
    sh = 4.0 * ((1 / 4.0) ** 6 - (1 / 4.0) ** 3)
    assert abs(_lj(1.0, 1.0, 2.0, sh, (1.9999, 0, 0))[0]) < 0.01
    assert abs(_lj(1.0, 1.0, 2.0, sh, (2.0, 0, 0))[0]) < 0.01
    assert _lj(1.0, 1.0, 2.0, sh, (10.0, 0, 0))[0] == 0.0
    # testLennardJones.py: eps = sig = 2
    assert abs(_lj(2.0, 2.0, math.inf, 0.0, (2.0, 0, 0))[0]) < 1e-12
    assert _lj(2.0, 2.0, math.inf, 0.0, (2 * 2 ** (1 / 6), 0, 0))[0] == pytest.approx(-2.0)


def test_polymer_melt_step0_matches_result_dat():
    pos, bonds, box, gold = load_polymer40k()
    s = Sim(oracle_lib(), box, 0.3, cell_grid(box, 1.12, 0.3))
    s.add(np.arange(1, len(pos) + 1), pos)
    s.decompose()
    s.vl(1.42)
    s.lj(0, 0, 1.0, 1.0, 1.12, 0.0)
    s.bonds(bonds)
    s.fene(30.0, 0.0, 1.5)
    assert round(s.energy(_abi.IA_LJ), 3) == gold["epair"]
    assert round(s.energy(_abi.IA_FENE), 3) == gold["ebond"]
    P = (s.virial(_abi.IA_LJ) + s.virial(_abi.IA_FENE)) / (3.0 * np.prod(box))
    assert round(P, 5) == gold["P"]


def _brute_pairs(pos, box, cut):
    n = len(pos)
    d = pos[:, None, :] - pos[None, :, :]
    d -= np.round(d / box) * box
    r2 = np.sum(d * d, -1)
    iu = np.triu_indices(n, 1)
    return int(np.sum(r2[iu] <= cut * cut))


def test_verlet_list_complete_vs_brute_force():
    # PTestVerletList.cpp: random particles, list size == N^2 count
    rng = np.random.Generator(np.random.PCG64(11))
    box = np.array([10.0, 11.0, 12.0])
    pos = rng.uniform(0, 1, size=(216, 3)) * box
    rc, skin = 1.5, 0.001
    s = Sim(oracle_lib(), box, skin, cell_grid(box, rc, skin))
    s.add(np.arange(216), pos)
    s.decompose()
    s.vl(rc)
    assert s.vl_size() == _brute_pairs(pos, box, rc + skin)
    # and on the 2048-particle LJ fixture
    pid, p2, _, b2 = load_lj2048()
    s2 = Sim(oracle_lib(), b2, 0.3, cell_grid(b2, 2.5, 0.3))
    s2.add(pid, p2)
    s2.decompose()
    s2.vl(2.5)
    folded = p2 - np.floor(p2 / b2) * b2
    assert s2.vl_size() == _brute_pairs(folded, b2, 2.8)


def test_pair_digest_matches_the_exported_pairs():
    """espp_vl_digest is the order-independent digest of the exported id pairs, it tells
    apart lists that differ by one pair, and it does not depend on the list order."""
    pid, pos, vel, box = load_lj2048()
    s = Sim(oracle_lib(), box, 0.3, cell_grid(box, 2.5, 0.3))
    s.add(pid, pos, vel)
    s.decompose()
    s.vl(2.5)
    pairs = s.pairs()
    d = s.digest()
    assert d == pair_digest(pairs)
    assert d == pair_digest(pairs[::-1][:, ::-1])
    assert d[0] == s.vl_size() == len(pairs)
    assert pair_digest(pairs[1:]) != d
    swapped = pairs.copy()
    swapped[0, 1] += 1
    assert pair_digest(swapped)[1:] != d[1:]


def test_nve_energy_conserved():
    pos, box = lattice(8, 0.8442, 0.05, seed=1)
    vel = mb_velocities(len(pos), 1.0, seed=2)
    s = Sim(oracle_lib(), box, 0.3, cell_grid(box, 2.5, 0.3))
    s.add(np.arange(len(pos)), pos, vel)
    s.decompose()
    s.vl(2.5)
    s.lj(0, 0, 1.0, 1.0, 2.5, 4.0 * (2.5 ** -12 - 2.5 ** -6))
    s.integrator(0.002)
    s.run(0)
    e0 = s.energy(_abi.IA_LJ) + 0.5 * s.kinetic()[0]
    s.run(200)
    e1 = s.energy(_abi.IA_LJ) + 0.5 * s.kinetic()[0]
    assert abs(e1 - e0) / len(pos) < 2e-4
    assert s.num_resorts() > 0


def test_langevin_thermalises_and_excludes():
    # testLangevinThermostat.py: an excluded particle keeps its velocity, others move
    pos, box = lattice(6, 0.5, 0.05, seed=3)
    n = len(pos)
    s = Sim(oracle_lib(), box, 0.3, cell_grid(box, 2.5, 0.3), seed=99)
    s.add(np.arange(n), pos, np.zeros((n, 3)))
    s.decompose()
    s.integrator(0.005)
    s.langevin(1.0, 2.0, excl=[0])
    s.run(400)
    _, v, _, _ = s.particles(np.arange(n))
    assert np.all(v[0] == 0.0)
    T = np.sum(v[1:] ** 2) / (3 * (n - 1))
    assert 1.4 < T < 2.6


def test_capforce_limits_total_force():
    pos, box = lattice(6, 1.2, 0.2, seed=5)
    n = len(pos)
    s = Sim(oracle_lib(), box, 0.3, cell_grid(box, 1.12246, 0.3))
    s.add(np.arange(n), pos)
    s.decompose()
    s.vl(1.12246)
    s.lj(0, 0, 1.0, 1.0, 1.12246, 1.0)
    s.capforce(_abi.CAP_ABS, 5.0)
    s.integrator(0.001)
    s.run(0)
    f = s.particles(np.arange(n))[2]
    assert np.max(np.linalg.norm(f, axis=1)) <= 5.0 + 1e-12


def test_tabulated_polymer_melt_step0_matches_result_dat(tmp_path):
    """testsuite/tabulated/result.dat, run with tabulated potentials: Akima tables of LJ
    and FENE written as polymer_melt_tabulated.py writes them."""
    from simdriver import polymer_tab_tables
    pos, bonds, box, gold = load_polymer40k()
    lib = oracle_lib()
    (rl, el, fl), (rf, ef, ff), _, _ = polymer_tab_tables(tmp_path, lib)
    s = Sim(lib, box, 0.3, cell_grid(box, 1.12, 0.3))
    s.add(np.arange(1, len(pos) + 1), pos)
    s.decompose()
    s.vl(1.42)
    s.bonds(bonds)
    call = _abi.call
    call(lib, "espp_tab_pair_set", s.h, 0, 0, 2, len(rl), _abi.dptr(rl), _abi.dptr(el),
         _abi.dptr(fl), 1.12, 0.0)
    call(lib, "espp_tab_bond_set", s.h, 2, len(rf), _abi.dptr(rf), _abi.dptr(ef),
         _abi.dptr(ff), math.inf, 0.0)
    g = gold["tabulated"]
    assert round(s.energy(_abi.IA_TAB_PAIR), 3) == g["epair"]
    assert round(s.energy(_abi.IA_TAB_BOND), 3) == g["ebond"]
    # The printed pressure of that run (3.80758) is not reproduced: the pair and bond
    # virials of these tables give 4.07021 (4.09383 linear, 4.08576 cubic), and the
    # angular term of the reference's run vanishes analytically (d12.F12 + d32.F32 = 0 in
    # FixedTripleListInteractionTemplate::computeVirial).  The pin is the two energies;
    # the tabulated virial is held to the analytic one within the interpolation error.
    P = (s.virial(_abi.IA_TAB_PAIR) + s.virial(_abi.IA_TAB_BOND)) / (3.0 * np.prod(box))
    assert abs(P - gold["P"]) < 0.02


def test_rdf_of_lj_fluid_is_normalised():
    """RadialDistrF on the 2048-particle LJ fixture: zero inside the core, first peak near
    2^(1/6), and g(r) -> 1 at long range (RadialDistrF.cpp:136-146 normalisation)."""
    pid, pos, _, box = load_lj2048()
    s = Sim(oracle_lib(), box, 0.3, cell_grid(box, 2.5, 0.3))
    s.add(pid, pos)
    s.decompose()
    g = np.zeros(100)
    _abi.call(oracle_lib(), "espp_rdf", s.h, 100, _abi.dptr(g))
    dr = box[1] / 2 / 100
    r = (np.arange(100) + 0.5) * dr
    assert np.all(g[r < 0.8] == 0.0)
    assert 1.0 < r[np.argmax(g)] < 1.25 and g.max() > 2.0
    assert abs(np.mean(g[(r > 4.5) & (r < 6.5)]) - 1.0) < 0.05


def _melt_with_angles(lib, prec=_abi.PREC_FP64, cosine=True, table=None):
    pos, bonds, box, gold, angles = load_polymer40k(angles=True)
    ids = np.arange(1, len(pos) + 1)
    s = Sim(lib, box, 0.3, cell_grid(box, 1.12, 0.3), precision=prec, seed=3)
    s.add(ids, pos)
    s.decompose()
    s.vl(1.42)
    s.lj(0, 0, 1.0, 1.0, 1.12, 0.0)
    s.bonds(bonds)
    s.fene(30.0, 0.0, 1.5)
    s.triples(angles)
    if cosine:
        s.cosine(1.5, 3.1415926)
    if table is not None:
        s.tab_angle(*table)
    s.integrator(0.002)
    return s, ids


def test_tabulated_angular_reproduces_cosine():
    """TabulatedAngular (TabulatedAngular.hpp:75-113) with a cubic table of the Cosine
    potential gives Cosine's energy, virial and forces on the 40 000 angles of the melt to
    the interpolation accuracy; both together add up."""
    c, ids = _melt_with_angles(oracle_lib(), cosine=True)
    t, _ = _melt_with_angles(oracle_lib(), cosine=False, table=(3,) + cosine_angle_table())
    both, _ = _melt_with_angles(oracle_lib(), cosine=True, table=(3,) + cosine_angle_table())
    ec, et = c.energy(_abi.IA_COSINE), t.energy(_abi.IA_TAB_ANGLE)
    assert abs(et - ec) < 1e-9 * abs(ec)
    assert abs(t.virial(_abi.IA_TAB_ANGLE) - c.virial(_abi.IA_COSINE)) < 1e-6 * abs(ec)
    for s in (c, t, both):
        s.run(0)
    fc, ft, fb = c.particles(ids)[2], t.particles(ids)[2], both.particles(ids)[2]
    assert np.max(np.abs(ft - fc)) < 1e-6 * np.max(np.abs(fc))
    # with both interactions the angle part of the force is twice the Cosine one
    base, _ = _melt_with_angles(oracle_lib(), cosine=False)
    base.run(0)
    fn = base.particles(ids)[2]
    assert np.max(np.abs((fb - fn) - 2 * (fc - fn))) < 1e-6 * np.max(np.abs(fc - fn))


def _lj2048_msd_run(lib, prec=_abi.PREC_FP64, nsnap=6, every=20, key=_abi.CONF_UNFOLDED):
    pid, pos, vel, box = load_lj2048()
    s = Sim(lib, box, 0.3, cell_grid(box, 2.5, 0.3), precision=prec, seed=11)
    s.add(pid, pos, vel)
    s.decompose()
    s.vl(2.5)
    s.lj(0, 0, 1.0, 1.0, 2.5, 4.0 * (2.5 ** -12 - 2.5 ** -6))
    s.integrator(0.005)
    s.langevin(1.0, 1.0)
    c = s.confs(key, pid)
    for _ in range(nsnap):
        c.gather()
        s.run(every)
    return s, c, pid, box


def test_msd_oracle_matches_direct_evaluation():
    """MeanSquareDispl::compute / computeG3 of the oracle against a direct numpy evaluation
    of the reference's sums on the same snapshots, and the "unfolded" key against
    position + image * box of the same particles (ConfigsParticleDecomp.cpp:70-142)."""
    s, c, pid, box = _lj2048_msd_run(oracle_lib())
    assert c.size() == 6
    snaps = np.array([c.get(m) for m in range(6)])
    got = c.msd()
    want = msd_reference(snaps)
    assert got[0] == 0.0
    assert np.allclose(got, want, rtol=1e-12, atol=0)
    assert np.all(np.diff(got) > 0)  # displacement grows with the lag in a liquid
    for L in (1, 16, 100):
        assert np.allclose(c.msd_chain(L), msd_chain_reference(snaps, L), rtol=1e-10, atol=1e-15)
    pos, _, _, img = s.particles(pid)
    c.gather()
    last = c.get(6)
    assert np.array_equal(last, pos + img * np.asarray(box))
    with pytest.raises(RuntimeError, match="out-of-range"):
        c.get(7)
    call = _abi.call
    call(oracle_lib(), "espp_confs_clear", c.h)
    assert c.size() == 0
    c.push(snaps[2])
    assert np.array_equal(c.get(0), snaps[2])


def test_polymer_melt_step0_angle_energy_matches_result_dat():
    """testsuite/tabulated/result.dat step 0: eangle 32301.755 of FixedTripleListCosine
    (Cosine K=1.5, theta0=3.1415926) on the 40 000 angles of polymer_melt.start.
    The printed value is sum K (1 - cos(theta - theta0)) (to the printed digits:
    32301.7548), the form of an earlier Cosine; the current source has K (1 + cos(theta -
    theta0)) (src/interaction/Cosine.hpp:74), which the oracle follows.  The two sum to
    2 K per angle, so the oracle's energy pins the same angles: 2 K N - E = 32301.755."""
    pos, bonds, box, gold, angles = load_polymer40k(angles=True)
    s = Sim(oracle_lib(), box, 0.3, cell_grid(box, 1.12, 0.3))
    s.add(np.arange(1, len(pos) + 1), pos)
    s.decompose()
    s.triples(angles)
    s.cosine(1.5, 3.1415926)
    e = s.energy(_abi.IA_COSINE)
    assert round(2 * 1.5 * len(angles) - e, 3) == gold["eangle"]
    # the angular virial vanishes: d12.F12 + d32.F32 = 0 for any angular force
    assert abs(s.virial(_abi.IA_COSINE)) < 1e-6


def _lj2048_nve(capped=False):
    """The setup of test_vec_lennard_jones.py: 2048-particle fluid with velocities, VL
    cutoff 2.5, skin 0.3, dt 0.005; LJ(rc 2.5, shift 0) or LJCapped(rc 2^(1/6), caprad
    0.6, shift auto)."""
    pid, pos, vel, box = load_lj2048()
    s = Sim(oracle_lib(), box, 0.3, cell_grid(box, 2.5, 0.3))
    s.add(pid + 1, pos, vel)
    s.decompose()
    s.vl(2.5)
    if capped:
        rc = 2.0 ** (1.0 / 6.0)
        s.lj(0, 0, 1.0, 1.0, rc, 4.0 * (rc ** -12 - rc ** -6), caprad=0.6)
    else:
        s.lj(0, 0, 1.0, 1.0, 2.5, 0.0)
    s.integrator(0.005)
    return s


@pytest.mark.parametrize("capped", [False, True])
@pytest.mark.parametrize("steps", [10, 400])
def test_vec_twin_matches_classic(steps, capped):
    """The vec twin (SoA cells padded to 64-byte rows, packed half-shell candidates,
    padded neighbour rows, N3L force rows) against the classic AoS step on the 2048-particle
    fluid with velocities: the reference's test_vec_lennard_jones.py runs 10 NVE steps and
    asks |dx|^2 = 0 to 8 places; 400 steps take many re-sorts through both paths."""
    pid, pos, vel, box = load_lj2048()
    ids = pid + 1
    classic, vec = _lj2048_nve(capped), _lj2048_nve(capped)
    classic.run(steps)
    _abi.call(vec.lib, "espp_vec_run", vec.h, steps)
    a, b = classic.particles(ids), vec.particles(ids)
    unf = lambda p: p[0] + p[3] * box
    d2 = np.sum((unf(a) - unf(b)) ** 2, axis=1)
    assert np.max(d2) < (5e-9 if steps == 10 else 1e-12)
    assert np.max(np.abs(a[1] - b[1])) < 1e-6
    assert vec.step() == classic.step() == steps
    assert vec.num_resorts() == classic.num_resorts()
    if steps == 400:
        assert classic.num_resorts() > 5
        assert vec.builds() == classic.builds()
    # the AoS side is consistent after a vec run: energies over the rebuilt pair list
    assert vec.energy(_abi.IA_LJ) == pytest.approx(classic.energy(_abi.IA_LJ), rel=1e-9)


def test_vec_twin_refuses_what_it_does_not_restate():
    s = _lj2048_nve()
    s.capforce(_abi.CAP_ABS, [10.0, 10.0, 10.0])
    with pytest.raises(RuntimeError, match="restates Lennard-Jones, FENE, Cosine and Langevin"):
        _abi.call(s.lib, "espp_vec_run", s.h, 1)


def test_vec_twin_langevin_matches_classic():
    """Langevin (gamma 1, T 1.5) with one excluded particle: the vec twin's thermalize
    draws the same counter-based noise, so vec and classic runs agree to rounding."""
    pid, pos, vel, box = load_lj2048()
    ids = pid + 1
    classic, vec = _lj2048_nve(), _lj2048_nve()
    for s in (classic, vec):
        s.langevin(1.0, 1.5, excl=[5])
    classic.run(100)
    _abi.call(vec.lib, "espp_vec_run", vec.h, 100)
    a, b = classic.particles(ids), vec.particles(ids)
    assert np.max(np.abs((a[0] + a[3] * box) - (b[0] + b[3] * box))) < 1e-8
    assert vec.builds() == classic.builds()


def test_vec_twin_langevin_exclusion_keeps_a_free_particle_still():
    """test_vec_langevin_thermostat.py: three particles at rest without interactions; the
    excluded one does not move, the thermostat moves the other two."""
    box = np.array([10.0, 10.0, 10.0])
    s = Sim(oracle_lib(), box, 0.3, cell_grid(box, 1.0, 0.3))
    s.add(np.array([1, 2, 3]), np.array([[1.0, 1.0, 1.0], [5.0, 5.0, 5.0], [8.0, 2.0, 6.0]]))
    s.decompose()
    s.integrator(0.01)
    s.langevin(1.0, 1.0, excl=[1])
    before = s.particles(np.array([1, 2, 3]))[0]
    _abi.call(s.lib, "espp_vec_run", s.h, 10)
    after = s.particles(np.array([1, 2, 3]))[0]
    assert np.array_equal(before[0], after[0])
    assert np.all(before[1:] != after[1:])


def test_vec_twin_runs_interleave_with_classic_runs():
    """Consecutive vec runs keep their SoA array and list; a classic run after them, and
    observables in between, see the particles where the vec run left them."""
    pid, pos, vel, box = load_lj2048()
    ids = pid + 1
    classic, vec = _lj2048_nve(), _lj2048_nve()
    for n in (150, 150):
        classic.run(n)
        _abi.call(vec.lib, "espp_vec_run", vec.h, n)
        assert vec.energy(_abi.IA_LJ) == pytest.approx(classic.energy(_abi.IA_LJ), rel=1e-9)
        assert vec.vl_size() > 0
    classic.run(50)
    vec.run(50)
    a, b = classic.particles(ids), vec.particles(ids)
    assert np.max(np.abs((a[0] + a[3] * box) - (b[0] + b[3] * box))) < 1e-8
    assert vec.step() == classic.step() == 350
    assert vec.builds() == classic.builds()


def test_vec_twin_matches_classic_on_the_polymer_melt():
    """test_vec_polymer_melt.py's check: the 40 000-bead melt with WCA (rc 2^(1/6), shift
    0), FENE(30, 0, 1.5) and Cosine(1.5, 3.1415926), skin 0.4, dt 0.005, 10 NVE steps from
    rest; vec and classic positions agree, |dx|^2 = 0 to 8 places."""
    pos, bonds, box, _, angles = load_polymer40k(angles=True)
    ids = np.arange(1, len(pos) + 1)
    rc = 2.0 ** (1.0 / 6.0)
    sims = []
    for _ in range(2):
        s = Sim(oracle_lib(), box, 0.4, cell_grid(box, rc, 0.4))
        s.add(ids, pos)
        s.decompose()
        s.vl(rc)
        s.lj(0, 0, 1.0, 1.0, rc, 0.0)
        s.bonds(bonds)
        s.fene(30.0, 0.0, 1.5)
        s.triples(angles)
        s.cosine(1.5, 3.1415926)
        s.integrator(0.005)
        sims.append(s)
    classic, vec = sims
    classic.run(10)
    _abi.call(vec.lib, "espp_vec_run", vec.h, 10)
    a, b = classic.particles(ids), vec.particles(ids)
    d2 = np.sum(((a[0] + a[3] * box) - (b[0] + b[3] * box)) ** 2, axis=1)
    assert np.max(d2) < 5e-9
    assert np.max(np.abs(a[1] - b[1])) < 1e-6
    for which in (_abi.IA_LJ, _abi.IA_FENE, _abi.IA_COSINE):
        assert vec.energy(which) == pytest.approx(classic.energy(which), rel=1e-9)


@pytest.mark.parametrize("steps", [10, 200])
def test_vec_list_equals_classic_list(steps):
    """verlet_list_buffer.py's check, classic AoS list against the vec twin's list: the
    same sorted id pairs after Langevin steps (both rebuilt on the same steps)."""
    classic, vec = _lj2048_nve(), _lj2048_nve()
    for s in (classic, vec):
        s.langevin(1.0, 1.0)
    classic.run(steps)
    _abi.call(vec.lib, "espp_vec_run", vec.h, steps)
    want = classic.pairs()
    n = ctypes.c_int64()
    _abi.call(vec.lib, "espp_vec_pairs", vec.h, 0, None, ctypes.byref(n))
    got = np.zeros((n.value, 2), np.int64)
    _abi.call(vec.lib, "espp_vec_pairs", vec.h, n.value,
              got.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(n))
    assert vec.builds() == classic.builds()
    assert len(got) == len(want) > 0
    assert np.array_equal(got, want)
