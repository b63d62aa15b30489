"""GPU parity against the FP64 oracle (both driven through the same C ABI)."""
import ctypes
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import (Sim, cell_grid, cosine_angle_table, cuda_lib, lattice, load_lj2048,
                       load_polymer40k, mb_velocities, msd_chain_reference, msd_reference,
                       oracle_lib)

pytestmark = pytest.mark.gpu


def _lj_setup(lib, prec, pid, pos, vel, box, rc=2.5, skin=0.3, shift=None, seed=7):
    s = Sim(lib, box, skin, cell_grid(box, rc, skin), precision=prec, seed=seed)
    s.add(pid, pos, vel)
    s.decompose()
    s.vl(rc)
    if shift is None:
        shift = 4.0 * ((1.0 / rc ** 2) ** 6 - (1.0 / rc ** 2) ** 3)
    s.lj(0, 0, 1.0, 1.0, rc, shift)
    return s


def _rel_rms(a, b):
    return math.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2))


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_lj2048_pairs_bit_exact(prec):
    pid, pos, vel, box = load_lj2048()
    o = _lj_setup(oracle_lib(), _abi.PREC_FP64, pid, pos, vel, box)
    g = _lj_setup(cuda_lib(), prec, pid, pos, vel, box)
    po, pg = o.pairs(), g.pairs()
    assert len(po) == len(pg) == o.vl_size() == g.vl_size()
    assert np.array_equal(po, pg)


def test_lj2048_forces_energy_fp64_and_mixed():
    pid, pos, vel, box = load_lj2048()
    o = _lj_setup(oracle_lib(), _abi.PREC_FP64, pid, pos, vel, box)
    g64 = _lj_setup(cuda_lib(), _abi.PREC_FP64, pid, pos, vel, box)
    gmx = _lj_setup(cuda_lib(), _abi.PREC_MIXED, pid, pos, vel, box)
    for s in (o, g64, gmx):
        s.integrator(0.005)
        s.run(0)
    fo = o.particles(pid)[2]
    f64 = g64.particles(pid)[2]
    fmx = gmx.particles(pid)[2]
    assert _rel_rms(f64, fo) < 1e-12
    assert _rel_rms(fmx, fo) < 1e-5
    eo = o.energy(_abi.IA_LJ)
    assert abs(g64.energy(_abi.IA_LJ) - eo) < 1e-10 * abs(eo)
    assert abs(gmx.energy(_abi.IA_LJ) - eo) < 1e-10 * abs(eo)
    wo = o.virial(_abi.IA_LJ)
    assert abs(g64.virial(_abi.IA_LJ) - wo) < 1e-10 * abs(wo)
    assert np.allclose(g64.virial_tensor(_abi.IA_LJ), o.virial_tensor(_abi.IA_LJ), rtol=1e-9,
                       atol=1e-9)


def test_polymer_melt_golden_step0():
    pos, bonds, box, gold = load_polymer40k()
    ids = np.arange(1, len(pos) + 1)
    for prec in (_abi.PREC_FP64, _abi.PREC_MIXED):
        s = Sim(cuda_lib(), box, 0.3, cell_grid(box, 1.12, 0.3), precision=prec)
        s.add(ids, pos)
        s.decompose()
        s.vl(1.42)
        s.lj(0, 0, 1.0, 1.0, 1.12, 0.0)
        s.bonds(bonds)
        s.fene(30.0, 0.0, 1.5)
        assert round(s.energy(_abi.IA_LJ), 3) == gold["epair"]
        assert round(s.energy(_abi.IA_FENE), 3) == gold["ebond"]
        P = (s.virial(_abi.IA_LJ) + s.virial(_abi.IA_FENE)) / (3.0 * np.prod(box))
        assert round(P, 5) == gold["P"]


@pytest.mark.parametrize("langevin", [False, True])
def test_lj_short_run_matches_oracle(langevin):
    pos, box = lattice(12, 0.8442, 0.05, seed=1)
    vel = mb_velocities(len(pos), 1.0, seed=2)
    pid = np.arange(len(pos))
    sims = [_lj_setup(oracle_lib(), _abi.PREC_FP64, pid, pos, vel, box),
            _lj_setup(cuda_lib(), _abi.PREC_FP64, pid, pos, vel, box),
            _lj_setup(cuda_lib(), _abi.PREC_MIXED, pid, pos, vel, box)]
    for s in sims:
        s.integrator(0.005)
        if langevin:
            s.langevin(1.0, 1.0)
        s.run(20)
    ref = sims[0].particles(pid)
    for s, tol in ((sims[1], 1e-9), (sims[2], 1e-5)):
        got = s.particles(pid)
        assert np.max(np.abs(got[0] - ref[0])) < tol
        assert np.array_equal(got[3], ref[3])
        assert _rel_rms(got[1], ref[1]) < tol
        assert s.step() == sims[0].step() == 20
    assert sims[1].num_resorts() == sims[0].num_resorts()


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_graph_loop_matches_host_loop(prec, monkeypatch):
    """The captured WHILE/IF step-loop graph and the host-driven loop run the same kernels
    in the same order: identical trajectories bit for bit, re-sorts included."""
    pos, box = lattice(16, 0.8442, 0.05, seed=1)
    vel = mb_velocities(len(pos), 1.5, seed=2)
    pid = np.arange(len(pos))
    sims = []
    for graph in ("0", "1"):
        monkeypatch.setenv("ESPP_B200_GRAPH", graph)
        s = _lj_setup(cuda_lib(), prec, pid, pos, vel, box)
        s.integrator(0.005)
        s.langevin(1.0, 1.5)
        s.run(60)
        s.run(7)
        sims.append(s)
    a, b = sims[0].particles(pid), sims[1].particles(pid)
    for k in range(4):
        assert np.array_equal(a[k], b[k])
    assert sims[0].num_resorts() == sims[1].num_resorts()
    assert sims[0].builds() == sims[1].builds() > 2
    assert sims[0].step() == sims[1].step() == 67


@pytest.mark.parametrize("tpp", [1, 2, 4, 8])
def test_mixed_forces_every_threads_per_particle(tpp):
    pid, pos, vel, box = load_lj2048()
    o = _lj_setup(oracle_lib(), _abi.PREC_FP64, pid, pos, vel, box)
    o.integrator(0.005)
    o.run(0)
    fo = o.particles(pid)[2]
    got = []
    for _ in range(2):
        g = _lj_setup(cuda_lib(), _abi.PREC_MIXED, pid, pos, vel, box)
        _abi.call(g.lib, "espp_set_tpp", g.h, tpp)
        g.integrator(0.005)
        g.run(0)
        got.append(g.particles(pid)[2])
    assert np.array_equal(got[0], got[1])  # deterministic for a fixed setting
    assert _rel_rms(got[0], fo) < 1e-5


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_large_cells_pairs_and_forces(prec):
    """3x3x3 cells of ~76 particles: the Verlet build walks the cell in groups of 32 and
    the in-cell sort takes its fallback path; the pair set stays the reference's."""
    pid, pos, vel, box = load_lj2048()
    sims = []
    for lib, p in ((oracle_lib(), _abi.PREC_FP64), (cuda_lib(), prec)):
        s = Sim(lib, box, 0.3, [3, 3, 3], precision=p)
        s.add(pid, pos, vel)
        s.decompose()
        s.vl(2.5)
        s.lj(0, 0, 1.0, 1.0, 2.5, 4.0 * (2.5 ** -12 - 2.5 ** -6))
        s.integrator(0.005)
        s.run(10)
        sims.append(s)
    assert np.array_equal(sims[0].pairs(), sims[1].pairs())
    ro, rg = sims[0].particles(pid), sims[1].particles(pid)
    assert np.max(np.abs(rg[0] - ro[0])) < (1e-9 if prec == _abi.PREC_FP64 else 1e-5)


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_polymer_melt_langevin_run_matches_oracle(prec):
    """40 000-bead ring melt: WCA (rc 1.12, shift 0) + FENE + Langevin, 15 steps."""
    pos, bonds, box, gold = load_polymer40k()
    ids = np.arange(1, len(pos) + 1)
    sims = []
    for lib, p in ((oracle_lib(), _abi.PREC_FP64), (cuda_lib(), prec)):
        s = Sim(lib, box, 0.3, cell_grid(box, 1.12, 0.3), precision=p, seed=54321)
        s.add(ids, pos)
        s.decompose()
        s.vl(1.42)
        s.lj(0, 0, 1.0, 1.0, 1.12, 0.0)
        s.bonds(bonds)
        s.fene(30.0, 0.0, 1.5)
        s.integrator(0.01)
        s.langevin(1.0, 1.0)
        s.run(15)
        sims.append(s)
    ro, rg = sims[0].particles(ids), sims[1].particles(ids)
    tol = 1e-9 if prec == _abi.PREC_FP64 else 2e-5
    assert np.max(np.abs(rg[0] - ro[0])) < tol
    assert np.array_equal(rg[3], ro[3])
    for which in (_abi.IA_LJ, _abi.IA_FENE):
        eo, eg = sims[0].energy(which), sims[1].energy(which)
        assert abs(eg - eo) < (1e-9 if prec == _abi.PREC_FP64 else 1e-5) * abs(eo)


def test_multitype_lj_with_exclusions():
    pid, pos, vel, box = load_lj2048()
    types = (pid % 3).astype(np.int32)
    excl = np.array([[int(pid[k]), int(pid[k + 1])] for k in range(0, 400, 2)])
    sims = []
    for lib, p in ((oracle_lib(), _abi.PREC_FP64), (cuda_lib(), _abi.PREC_FP64),
                   (cuda_lib(), _abi.PREC_MIXED)):
        s = Sim(lib, box, 0.3, cell_grid(box, 2.5, 0.3), precision=p)
        s.add(pid, pos, vel, types=types)
        s.decompose()
        s.vl(2.5, excl=excl)
        s.lj(0, 0, 1.0, 1.0, 2.5, 0.0)
        s.lj(0, 1, 1.5, 0.9, 2.2, 0.0)
        s.lj(1, 1, 0.7, 1.1, 2.5, 0.0)
        s.lj(2, 2, 1.2, 1.0, 2.0, 0.0)
        # pairs (0,2) and (1,2) left unset: no interaction, as in the reference's table
        s.integrator(0.005)
        s.run(5)
        sims.append(s)
    for s in sims[1:]:
        assert np.array_equal(s.pairs(), sims[0].pairs())
    ex = set(map(tuple, np.sort(excl, axis=1)))
    assert not ex & set(map(tuple, sims[0].pairs()))
    ro = sims[0].particles(pid)
    assert np.max(np.abs(sims[1].particles(pid)[0] - ro[0])) < 1e-9
    assert np.max(np.abs(sims[2].particles(pid)[0] - ro[0])) < 1e-5
    eo = sims[0].energy(_abi.IA_LJ)
    assert abs(sims[1].energy(_abi.IA_LJ) - eo) < 1e-9 * abs(eo)


@pytest.mark.parametrize("mode,cap", [(_abi.CAP_ABS, 20.0), (_abi.CAP_COMPONENT, [15.0, 10.0, 5.0])])
def test_capforce_and_capped_lj(mode, cap):
    pos, box = lattice(10, 1.1, 0.25, seed=7)   # dense, overlapping start
    pid = np.arange(len(pos))
    sims = []
    for lib, p in ((oracle_lib(), _abi.PREC_FP64), (cuda_lib(), _abi.PREC_FP64),
                   (cuda_lib(), _abi.PREC_MIXED)):
        s = Sim(lib, box, 0.3, cell_grid(box, 2 ** (1 / 6), 0.3), precision=p)
        s.add(pid, pos)
        s.decompose()
        s.vl(2 ** (1 / 6))
        s.lj(0, 0, 1.0, 1.0, 2 ** (1 / 6), 1.0, caprad=0.9)
        s.capforce(mode, cap)
        s.integrator(0.002)
        s.langevin(0.5, 1.0)
        s.run(10)
        sims.append(s)
    ro = sims[0].particles(pid)
    assert np.max(np.abs(sims[1].particles(pid)[0] - ro[0])) < 1e-9
    assert np.max(np.abs(sims[2].particles(pid)[0] - ro[0])) < 1e-5
    f = sims[1].particles(pid)[2]
    if mode == _abi.CAP_ABS:
        assert np.max(np.linalg.norm(f, axis=1)) <= cap * (1 + 1e-12)
    else:
        assert np.all(np.abs(f) <= np.array(cap) * (1 + 1e-12))


def _replica(lib, n_side, rho, T, seed, prec):
    pos, box = lattice(n_side, rho, 0.05, seed=seed)
    vel = mb_velocities(len(pos), T, seed=seed + 100)
    s = _lj_setup(lib, prec, np.arange(len(pos)), pos, vel, box, seed=seed)
    s.integrator(0.005)
    s.langevin(1.0, T)
    return s


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_batch_run_matches_individual_runs(prec):
    """One graph launch stepping 4 replicas of different sizes and temperatures gives
    each replica exactly the trajectory of espp_run on it alone."""
    import ctypes
    specs = [(9, 0.8442, 0.8, 1), (12, 0.8442, 1.2, 2), (14, 0.8, 1.6, 3), (10, 0.85, 2.0, 4)]
    lib = cuda_lib()
    solo = [_replica(lib, *sp, prec) for sp in specs]
    for s in solo:
        s.run(40)
        s.run(25)
    rep = [_replica(lib, *sp, prec) for sp in specs]
    arr = (ctypes.c_void_p * len(rep))(*[s.h.value for s in rep])
    b = ctypes.c_void_p()
    _abi.call(lib, "espp_batch_create", arr, len(rep), ctypes.byref(b))
    try:
        _abi.call(lib, "espp_batch_run", b, 40)
        _abi.call(lib, "espp_batch_run", b, 25)
    finally:
        lib.espp_batch_destroy(b)
    for a, c, sp in zip(solo, rep, specs):
        ids = np.arange(sp[0] ** 3)
        pa, pc = a.particles(ids), c.particles(ids)
        for k in range(4):
            assert np.array_equal(pa[k], pc[k])
        assert a.num_resorts() == c.num_resorts() and a.step() == c.step() == 65
        assert a.builds() == c.builds()


def test_parallel_tempering_api_runs_and_exchanges():
    import random
    import espressopp_b200 as espressopp
    pt = espressopp.ParallelTempering(NumberOfSystems=4, RNG=random.Random(7))
    for i in range(pt.getNumberOfSystems()):
        pt.startDefiningSystem(i)
        x, y, z, Lx, Ly, Lz = espressopp.tools.lattice.createCubic(1000 + 200 * i, 0.8442,
                                                                    perfect=False)
        system = espressopp.System()
        system.rng = espressopp.esutil.RNG(100 + i)
        system.bc = espressopp.bc.OrthorhombicBC(system.rng, (Lx, Ly, Lz))
        system.skin = 0.3
        cg = espressopp.tools.decomp.cellGrid((Lx, Ly, Lz), (1, 1, 1), 2.5, 0.3)
        system.storage = espressopp.storage.DomainDecomposition(system, (1, 1, 1), cg)
        system.storage.addParticles([[k, espressopp.Real3D(x[k], y[k], z[k])]
                                     for k in range(len(x))], "id", "pos")
        system.storage.decompose()
        vl = espressopp.VerletList(system, cutoff=2.5)
        lj = espressopp.interaction.VerletListLennardJones(vl)
        lj.setPotential(0, 0, espressopp.interaction.LennardJones(1.0, 1.0, 2.5, 0.0))
        system.addInteraction(lj)
        integ = espressopp.integrator.VelocityVerlet(system)
        integ.dt = 0.005
        lang = espressopp.integrator.LangevinThermostat(system)
        lang.gamma = 1.0
        lang.temperature = 0.7 + 0.4 * i
        integ.addExtension(lang)
        pt.setIntegrator(integ, lang)
        pt.setAnalysisE(lj)
        pt.setAnalysisT(espressopp.analysis.Temperature(system))
        pt.setAnalysisNPart(espressopp.analysis.NPart(system))
        pt.endDefiningSystem(i)
    for _ in range(3):
        pt.run(50)
        before = [th.temperature for th in pt._thermostat]
        measured = pt._multisystem.runAnalysisTemperature()
        decisions = pt.exchange()
        assert len(decisions) >= 1
        # the reference gives each exchanged thermostat the other replica's measured T
        for m, n, _, _, ok in decisions:
            if ok:
                assert pt._thermostat[n].temperature == pytest.approx(measured[m], rel=1e-12)
                assert pt._thermostat[m].temperature == pytest.approx(measured[n], rel=1e-12)
            else:
                assert pt._thermostat[n].temperature == before[n]
    temps = pt._multisystem.runAnalysisTemperature()
    assert all(0.05 < t < 10.0 for t in temps)


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_tabulated_angular_matches_oracle(prec, tmp_path):
    """FixedTripleListTabulatedAngular on the 40 000-bead melt (an Akima table of a bent
    angle potential, with Cosine acting too): energy, virial and forces against the oracle,
    then a short Langevin run; the Python classes read the same table from a file."""
    from test_oracle import _melt_with_angles
    th = np.linspace(0.0, math.pi, 181)
    e = 2.0 * (np.cos(th) - np.cos(2.0)) ** 2
    f = 4.0 * (np.cos(th) - np.cos(2.0)) * np.sin(th)
    sims = [_melt_with_angles(lib, p, cosine=True, table=(2, th, e, f))[0]
            for lib, p in ((oracle_lib(), _abi.PREC_FP64), (cuda_lib(), prec))]
    o, g = sims
    ids = np.arange(1, 40001)
    eo = o.energy(_abi.IA_TAB_ANGLE)
    assert abs(g.energy(_abi.IA_TAB_ANGLE) - eo) < 1e-9 * abs(eo)
    wo = o.virial(_abi.IA_TAB_ANGLE)
    assert abs(g.virial(_abi.IA_TAB_ANGLE) - wo) < 1e-9 * abs(eo)
    for s in sims:
        s.run(0)
    tol = 1e-12 if prec == _abi.PREC_FP64 else 1e-5
    assert _rel_rms(g.particles(ids)[2], o.particles(ids)[2]) < tol
    for s in sims:
        s.langevin(1.0, 1.0)
        s.run(20)
    assert np.max(np.abs(g.particles(ids)[0] - o.particles(ids)[0])) < (
        1e-9 if prec == _abi.PREC_FP64 else 1e-4)
    import espressopp_b200 as espressopp
    path = tmp_path / "angle.tab"
    with open(path, "w") as fh:
        for a, b, c in zip(th, e, f):
            fh.write("%.17g %.17g %.17g\n" % (a, b, c))
    pot = espressopp.interaction.TabulatedAngular(2, str(path))
    assert pot.computeEnergy(1.3) == pytest.approx(2.0 * (math.cos(1.3) - math.cos(2.0)) ** 2,
                                                   rel=1e-3)


def test_kinetic_tensor_matches_oracle():
    """sum of mass * Tensor(v, v) (PressureTensor.hpp:60-70) on the GPU against the oracle;
    its trace is the kinetic sum of Temperature."""
    pid, pos, vel, box = load_lj2048()
    outs = []
    for lib in (oracle_lib(), cuda_lib()):
        s = _lj_setup(lib, _abi.PREC_FP64, pid, pos, vel, box)
        t = np.zeros(6)
        _abi.call(lib, "espp_kinetic_tensor", s.h, _abi.dptr(t))
        outs.append((t, s.kinetic()))
    (to, ko), (tg, kg) = outs
    assert np.allclose(tg, to, rtol=1e-12, atol=1e-12 * np.abs(to).max())
    assert abs(tg[:3].sum() - kg[0]) < 1e-12 * kg[0]


def test_msd_matches_oracle():
    """MeanSquareDispl::compute / computeG3 on the GPU against the oracle on the same
    snapshots (FP64, only the summation order differs), and GPU snapshots of the same
    Langevin run against the oracle's (ConfigsParticleDecomp.cpp:70-142)."""
    from test_oracle import _lj2048_msd_run
    so, co, pid, box = _lj2048_msd_run(oracle_lib())
    sg, cg_, _, _ = _lj2048_msd_run(cuda_lib())
    snaps_o = np.array([co.get(m) for m in range(co.size())])
    snaps_g = np.array([cg_.get(m) for m in range(cg_.size())])
    assert snaps_g.shape == snaps_o.shape
    assert np.max(np.abs(snaps_g - snaps_o)) < 1e-8
    # the same snapshots pushed into a GPU list: only the reduction order differs
    pg = sg.confs(_abi.CONF_UNFOLDED, pid)
    for m in range(len(snaps_o)):
        pg.push(snaps_o[m])
    assert np.allclose(pg.msd(), co.msd(), rtol=1e-12, atol=0)
    for L in (1, 16, 100):
        assert np.allclose(pg.msd_chain(L), co.msd_chain(L), rtol=1e-10, atol=1e-15)
    assert np.allclose(cg_.msd(), co.msd(), rtol=1e-6)
    pos, vel, _, img = sg.particles(pid)
    cg_.gather()
    assert np.array_equal(cg_.get(cg_.size() - 1), pos + img * np.asarray(box))
    cv = sg.confs(_abi.CONF_VELOCITY, pid)
    cv.gather()
    assert np.array_equal(cv.get(0), vel)
    bad = sg.confs(_abi.CONF_POSITION, np.array([10 ** 6], np.int64))
    with pytest.raises(RuntimeError, match="id"):
        bad.gather()


def test_msd_python_api():
    """analysis.MeanSquareDispl through the Python mirror on a small LJ fluid."""
    import espressopp_b200 as espressopp
    x, y, z, Lx, Ly, Lz = espressopp.tools.lattice.createCubic(1000, 0.8442, perfect=False)
    system = espressopp.System()
    system.rng = espressopp.esutil.RNG(5)
    system.bc = espressopp.bc.OrthorhombicBC(system.rng, (Lx, Ly, Lz))
    system.skin = 0.3
    cgrid = espressopp.tools.decomp.cellGrid((Lx, Ly, Lz), (1, 1, 1), 2.5, 0.3)
    system.storage = espressopp.storage.DomainDecomposition(system, (1, 1, 1), cgrid)
    system.storage.addParticles([[k, espressopp.Real3D(x[k], y[k], z[k])]
                                 for k in range(len(x))], "id", "pos")
    system.storage.decompose()
    vl = espressopp.VerletList(system, cutoff=2.5)
    lj = espressopp.interaction.VerletListLennardJones(vl)
    lj.setPotential(0, 0, espressopp.interaction.LennardJones(1.0, 1.0, 2.5))
    system.addInteraction(lj)
    integ = espressopp.integrator.VelocityVerlet(system)
    integ.dt = 0.005
    lang = espressopp.integrator.LangevinThermostat(system)
    lang.gamma = 1.0
    lang.temperature = 1.0
    integ.addExtension(lang)
    msd = espressopp.analysis.MeanSquareDispl(system, chainlength=10)
    for _ in range(5):
        msd.gather()
        integ.run(20)
    assert msd.size == 5
    snaps = np.array([[msd[m].getCoordinates(pid) for pid in range(1000)] for m in range(5)])
    got = msd.compute()
    assert np.allclose(got, msd_reference(snaps), rtol=1e-12, atol=0)
    assert np.allclose(msd.computeG3(), msd_chain_reference(snaps, 10), rtol=1e-10, atol=1e-15)
    assert msd.computeG2() == []
    msd.clear()
    assert msd.size == 0


@pytest.mark.parametrize("rdfN", [100, 1000, 20000])
def test_rdf_matches_oracle_bitwise(rdfN):
    """RadialDistrF: integer pair counts per bin are identical, so the normalised arrays
    are bitwise equal (RadialDistrF.cpp:47-150); the 20000-bin case uses global counts."""
    pid, pos, vel, box = load_lj2048()
    o = _lj_setup(oracle_lib(), _abi.PREC_FP64, pid, pos, vel, box)
    g = _lj_setup(cuda_lib(), _abi.PREC_FP64, pid, pos, vel, box)
    ho, hg = np.zeros(rdfN), np.zeros(rdfN)
    _abi.call(o.lib, "espp_rdf", o.h, rdfN, _abi.dptr(ho))
    _abi.call(g.lib, "espp_rdf", g.h, rdfN, _abi.dptr(hg))
    assert np.array_equal(ho, hg)
    # after a run the trajectories agree to ~1e-12, so at most a few pairs change bins
    for s in (o, g):
        s.integrator(0.005)
        s.run(40)
    _abi.call(o.lib, "espp_rdf", o.h, rdfN, _abi.dptr(ho))
    _abi.call(g.lib, "espp_rdf", g.h, rdfN, _abi.dptr(hg))
    dr = box[1] / 2 / rdfN
    r = (np.arange(rdfN) + 0.5) * dr
    one_pair = 1.0 / (2 * np.pi * dr * len(pid) ** 2 / np.prod(box) * (r * r + dr * dr / 12))
    assert np.sum(np.abs(ho - hg) / one_pair) <= 4.0


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_polymer_melt_with_angles_matches_oracle(prec):
    """FixedTripleListCosine with LJ and FENE on the 40 000-bead melt: the result.dat
    eangle at step 0, forces against the oracle, and a short Langevin run."""
    pos, bonds, box, gold, angles = load_polymer40k(angles=True)
    ids = np.arange(1, len(pos) + 1)
    sims = []
    for lib, p in ((oracle_lib(), _abi.PREC_FP64), (cuda_lib(), prec)):
        s = Sim(lib, box, 0.3, cell_grid(box, 1.12, 0.3), precision=p, seed=3)
        s.add(ids, pos)
        s.decompose()
        s.vl(1.42)
        s.lj(0, 0, 1.0, 1.0, 1.12, 0.0)
        s.bonds(bonds)
        s.fene(30.0, 0.0, 1.5)
        s.triples(angles)
        s.cosine(1.5, 3.1415926)
        sims.append(s)
    o, g = sims
    # result.dat prints sum K (1 - cos(theta - theta0)) = 2 K N - sum K (1 + cos(...))
    assert round(2 * 1.5 * len(angles) - g.energy(_abi.IA_COSINE), 3) == gold["eangle"]
    assert abs(g.energy(_abi.IA_COSINE) - o.energy(_abi.IA_COSINE)) < 1e-9 * gold["eangle"]
    for s in sims:
        s.integrator(0.002)
        s.run(0)
    tol = 1e-12 if prec == _abi.PREC_FP64 else 1e-5
    assert _rel_rms(g.particles(ids)[2], o.particles(ids)[2]) < tol
    for s in sims:
        s.langevin(1.0, 1.0)
        s.run(20)
    ref = o.particles(ids)
    got = g.particles(ids)
    assert np.max(np.abs(got[0] - ref[0])) < (1e-9 if prec == _abi.PREC_FP64 else 1e-4)


def test_fp32_probe_reports_a_plausible_peak():
    """The FP32 FMA probe behind the FLOP side of the roofline: a B200 sustains tens of
    TFLOP/s (148 SMs x 128 lanes x 2 FLOP x ~1.9 GHz = 72 TFLOP/s scalar)."""
    t = ctypes.c_double()
    _abi.call(cuda_lib(), "espp_fp32_peak", ctypes.byref(t))
    assert 20.0 < t.value < 400.0
