"""Host logic of the Python mirror driven through the CPU oracle library, which exports
the same C ABI as the CUDA library: here the mirror's own bookkeeping is under test, not
the GPU kernels (those are checked against the oracle in the gpu-marked tests)."""
import numpy as np
import pytest

import espressopp_b200 as espressopp
from espressopp_b200 import _lib
from simdriver import oracle_lib


@pytest.fixture
def on_oracle(monkeypatch):
    monkeypatch.setattr(_lib, "_lib", oracle_lib())


def _fluid(seed=5, n=1000):
    x, y, z, Lx, Ly, Lz = espressopp.tools.lattice.createCubic(
        n, 0.8442, perfect=False, RNG=espressopp.esutil.RNG(7))
    system = espressopp.System()
    system.rng = espressopp.esutil.RNG(seed)
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
    return system, integ


def test_configurations_trajectory(on_oracle):
    """analysis.Configurations (Configurations.cpp:44-110): folded and unfolded positions,
    velocities and forces by id, [n] counting back from the newest, capacity trimming."""
    system, integ = _fluid()
    L = np.asarray(system.bc.boxL)
    folded = espressopp.analysis.Configurations(system, vel=True, force=True)
    unfolded = espressopp.analysis.Configurations(system, folded=False, radius=True)
    for _ in range(4):
        integ.run(100)
        folded.gather()
        unfolded.gather()
    assert folded.size == unfolded.size == 4
    ids, pos, vel, frc, img = system.storage.getAll()
    assert np.any(img != 0)
    newest, u = folded[0], unfolded[0]
    assert newest is folded.back() and folded[4] is None
    for pid in (0, 17, 999):
        k = int(np.searchsorted(ids, pid))
        p = np.asarray(newest[pid])
        assert np.all(p >= 0.0) and np.all(p < L)
        assert np.allclose(np.asarray(u[pid]), pos[k] + img[k] * L, rtol=0, atol=1e-12)
        assert np.allclose(p, pos[k] - np.floor(pos[k] / L) * L, rtol=0, atol=1e-12)
        assert tuple(newest.getVelocities(pid)) == tuple(vel[k])
        assert tuple(newest.getForces(pid)) == tuple(frc[k])
        assert u.getRadius(pid) == 1.0
    with pytest.raises(RuntimeError):
        u.getVelocities(0)
    assert [c for c in folded] == folded.all() and folded.all()[-1] is newest
    folded.capacity = 2
    assert folded.size == 2 and folded[0] is newest
    folded.gather()
    assert folded.size == 2 and folded[1] is newest
    folded.capacity = -1
    assert folded.capacity == 2
    folded.clear()
    assert folded.size == 0


def test_checkpoint_resume_host_logic(on_oracle, tmp_path, monkeypatch):
    """The checkpoint/resume recipe of the Python mirror (RNG.saveState / loadState, a
    settable step, images through setImages) continues the uninterrupted Langevin run."""
    monkeypatch.chdir(tmp_path)
    full, integ_full = _fluid(2024)
    integ_full.run(120)
    integ_full.run(80)
    part, integ_part = _fluid(2024)
    integ_part.run(120)
    ids, pos, vel, _, img = part.storage.getAll()
    L = np.asarray(part.bc.boxL)
    t = np.floor(pos * (1.0 / L))
    pos, img = pos - t * L, img + t.astype(np.int32)
    part.rng.saveState(integ_part.step)
    # rebuild from the checkpoint in a fresh system keyed on the saved seed
    res = espressopp.System()
    res.rng = espressopp.esutil.RNG(99)
    res.rng.loadState("rng.120")
    assert res.rng.get_seed() == 2024
    res.bc = espressopp.bc.OrthorhombicBC(res.rng, tuple(L))
    res.skin = 0.3
    cgrid = espressopp.tools.decomp.cellGrid(tuple(L), (1, 1, 1), 2.5, 0.3)
    res.storage = espressopp.storage.DomainDecomposition(res, (1, 1, 1), cgrid)
    res.storage.addParticles([[int(ids[k]), espressopp.Real3D(pos[k]), espressopp.Real3D(vel[k])]
                              for k in range(len(ids))], "id", "pos", "v")
    res.storage.setImages(ids, img)
    res.storage.decompose()
    vl = espressopp.VerletList(res, cutoff=2.5)
    lj = espressopp.interaction.VerletListLennardJones(vl)
    lj.setPotential(0, 0, espressopp.interaction.LennardJones(1.0, 1.0, 2.5))
    res.addInteraction(lj)
    ri = espressopp.integrator.VelocityVerlet(res)
    ri.dt = 0.005
    lang = espressopp.integrator.LangevinThermostat(res)
    lang.gamma = 1.0
    lang.temperature = 1.0
    ri.addExtension(lang)
    ri.step = 120
    ri.run(80)
    a, b = full.storage.getAll(), res.storage.getAll()
    unf = lambda s: s[1] + s[4] * L
    assert np.max(np.abs(unf(a) - unf(b))) < 1e-8


def test_modify_particle_image_semantics(on_oracle):
    system, integ = _fluid()
    st = system.storage
    st.modifyParticle(3, "img", (2, -1, 4))
    assert tuple(st.getAll()[4][3]) == (2, -1, 4)
    st.modifyParticle(3, "pos", (1.0, 2.0, 3.0))
    _, pos, _, _, img = st.getAll()
    assert tuple(img[3]) == (0, 0, 0) and tuple(pos[3]) == (1.0, 2.0, 3.0)
    with pytest.raises(ValueError):
        st.modifyParticle(3, "q", 1.0)


def test_standard_systems_and_info(on_oracle, capsys):
    """standard_system.Minimal / LennardJones build what the reference builds, and
    tools.analyse.info / timers.show print from them."""
    system, integ = espressopp.standard_system.Minimal(200, (10.0, 10.0, 10.0), rc=2.5,
                                                       skin=0.3)
    ids, pos, vel, _, _ = system.storage.getAll()
    assert list(ids) == list(range(1, 201)) and np.all(vel == 0.0)
    assert np.all(pos >= 0.0) and np.all(pos < 10.0)
    assert system.getNumberOfInteractions() == 0
    integ.run(5)
    assert integ.step == 5
    # random positions overlap: the reference's recipe needs a capped warm-up before
    # stepping, so only the start-of-run forces are taken here
    system, integ = espressopp.standard_system.LennardJones(500, box=(9.0, 9.0, 9.0), rc=2.5,
                                                            temperature=1.0)
    assert system.getNumberOfInteractions() == 1
    integ.run(0)
    espressopp.tools.analyse.info(system, integ)
    espressopp.tools.timers.show(integ.getTimers())
    out = capsys.readouterr().out
    assert out.strip()
    vl = system.getInteraction(0).getVerletList()
    espressopp.tools.analyse.final_info(system, integ, vl, 1.0, 3.5)
    lines = capsys.readouterr().out.splitlines()
    # the reference's report (tools/analyse.py:66-76) after the timers block
    assert lines[-5] == "Total # of neighbors = %d" % vl.totalSize()
    assert lines[-4] == "Ave neighs/atom = %.1f" % (vl.totalSize() / 500.0)
    assert lines[-3] == "Neighbor list builds = %d" % vl.builds
    assert lines[-2] == "Integration steps = 0"
    assert lines[-1] == "CPUs = 1 CPU time per CPU = 2.50000"


def test_pressure_tensor_running_average(on_oracle):
    """PressureTensor.performMeasurement / getAverageValue: the running mean and the
    sample standard deviation of the measured tensors (PressureTensor.hpp:96-143)."""
    system, integ = _fluid()
    pt = espressopp.analysis.PressureTensor(system)
    assert pt.getAverageValue() == [0.0] * 12 and pt.getNumberOfMeasurements() == 0
    seen = []
    for _ in range(4):
        integ.run(20)
        seen.append(list(pt.compute()))
        pt.performMeasurement()
    avg = pt.getAverageValue()
    assert pt.getNumberOfMeasurements() == 4 and len(avg) == 12
    assert np.allclose(avg[:6], np.mean(seen, axis=0), rtol=1e-12, atol=1e-14)
    assert np.allclose(avg[6:], np.std(seen, axis=0, ddof=1), rtol=1e-9, atol=1e-14)
    pt.reset()
    pt.performMeasurement()
    assert pt.getNumberOfMeasurements() == 1 and all(np.isnan(avg_) for avg_ in
                                                     pt.getAverageValue()[6:])


def test_temperature_of_selected_types(on_oracle):
    """Temperature.add_type / remove_type (Temperature.hpp:104-141): only the selected
    types count; with none selected every particle does; no selected particle gives
    sumT / (3 * 0) = nan; getEkin is half the last sum of m v^2."""
    x, y, z, Lx, Ly, Lz = espressopp.tools.lattice.createCubic(
        512, 0.8442, perfect=False, RNG=espressopp.esutil.RNG(7))
    system = espressopp.System()
    system.rng = espressopp.esutil.RNG(5)
    system.bc = espressopp.bc.OrthorhombicBC(system.rng, (Lx, Ly, Lz))
    system.skin = 0.3
    cgrid = espressopp.tools.decomp.cellGrid((Lx, Ly, Lz), (1, 1, 1), 2.5, 0.3)
    system.storage = espressopp.storage.DomainDecomposition(system, (1, 1, 1), cgrid)
    types = [1 if k % 5 == 0 else (70 if k % 7 == 0 else 0) for k in range(len(x))]
    system.storage.addParticles([[k, espressopp.Real3D(x[k], y[k], z[k]), types[k]]
                                 for k in range(len(x))], "id", "pos", "type")
    system.storage.decompose()
    integ = espressopp.integrator.VelocityVerlet(system)
    integ.dt = 0.005
    lang = espressopp.integrator.LangevinThermostat(system)
    lang.gamma = 1.0
    lang.temperature = 1.0
    integ.addExtension(lang)
    integ.run(30)
    st = system.storage
    T = espressopp.analysis.Temperature(system)
    ids, _, vel, _, _ = st.getAll()
    typ = np.array([types[int(p)] for p in ids])
    v2 = np.sum(vel * vel, axis=1)
    all_T = float(np.sum(v2)) / (3 * len(ids))
    assert T.compute() == pytest.approx(all_T, rel=1e-12)
    assert T.getEkin() == pytest.approx(0.5 * float(np.sum(v2)), rel=1e-12)
    T.add_type(1)
    sel = typ == 1
    assert T.compute() == pytest.approx(float(np.sum(v2[sel])) / (3 * sel.sum()), rel=1e-12)
    T.add_type(70)  # a type id beyond the 64-bit mask of the device reduction
    sel = (typ == 1) | (typ == 70)
    assert T.compute() == pytest.approx(float(np.sum(v2[sel])) / (3 * sel.sum()), rel=1e-12)
    assert T.remove_type(1) and T.remove_type(70) and not T.remove_type(1)
    assert T.compute() == pytest.approx(all_T, rel=1e-12)
    T.add_type(3)  # no particle of type 3
    assert np.isnan(T.compute())


def test_named_interactions(on_oracle):
    """System.py:134-192: interactions added under a name are found, listed and removed by
    it; a repeated name, an unknown name and an index out of range are errors, and the
    names above a removed interaction move down with it.  The device holds one parameter
    table per interaction kind, so a second interaction of a kind is refused."""
    system, integ = _fluid(n=512)
    lj0 = system.getInteraction(0)
    fpl = espressopp.FixedPairList(system.storage)
    fpl.addBonds([(0, 1), (2, 3)])
    fene = espressopp.interaction.FixedPairListFENE(
        system, fpl, espressopp.interaction.FENE(K=30.0, r0=0.0, rMax=1.5))
    cos_ = espressopp.interaction.FixedTripleListCosine(
        system, espressopp.FixedTripleList(system.storage),
        espressopp.interaction.Cosine(K=1.5, theta0=0.0))
    system.addInteraction(fene, "bonds")
    system.addInteraction(cos_, "angles")
    with pytest.raises(RuntimeError, match="already defined"):
        system.addInteraction(cos_, "bonds")
    lj1 = espressopp.interaction.VerletListLennardJones(lj0.getVerletList())
    with pytest.raises(RuntimeError, match="one interaction of each kind"):
        system.addInteraction(lj1)
    assert system.getNumberOfInteractions() == 3
    assert system.getInteractionByName("angles") is cos_
    assert system.getNameOfInteraction(1) == "bonds" and system.getNameOfInteraction(0) is None
    assert set(system.getAllInteractions()) == {"bonds", "angles"}
    assert fene.computeEnergy() > 0.0
    system.removeInteractionByName("bonds")
    assert system.getNumberOfInteractions() == 2
    assert system.getNameOfInteraction(1) == "angles"
    assert system.getInteractionByName("angles") is cos_
    with pytest.raises(RuntimeError, match="not found"):
        system.removeInteractionByName("bonds")
    with pytest.raises(RuntimeError, match="does not exist"):
        system.getInteraction(2)
    integ.run(10)
    system.integrator = integ
    assert system.integrator is integ


def test_fixed_pair_list_longtime_max_and_remove(on_oracle):
    """FixedPairList (FixedPairList.py:85-148, FixedPairList.cpp:82-86 and 167-324): the
    long-time maximum bond is 0 before a force pass and the longest bond after it, a reset
    sets it to 0, getAllBonds lists every (pid1 < pid2) pair, remove empties the list;
    FixedTripleList.remove likewise."""
    system, integ = _fluid(n=512)
    fpl = espressopp.FixedPairList(system.storage)
    fpl.addBonds([(1, 0), (2, 3), (10, 11)])
    assert fpl.getAllBonds() == [(0, 1), (2, 3), (10, 11)]
    fene = espressopp.interaction.FixedPairListFENE(
        system, fpl, espressopp.interaction.FENE(K=30.0, r0=0.0, rMax=2.5))
    system.addInteraction(fene)
    assert fpl.getLongtimeMaxBond() == 0.0
    integ.run(0)
    ids, pos = system.storage.getAll()[:2]
    L = np.asarray(system.bc.boxL)
    d = np.array([pos[np.searchsorted(ids, a)] - pos[np.searchsorted(ids, b)]
                  for a, b in fpl.getAllBonds()])
    d -= L * np.round(d / L)
    longest = float(np.sqrt(np.max(np.sum(d * d, axis=1))))
    assert abs(fpl.getLongtimeMaxBond() - longest) < 1e-12 * longest
    assert fpl.getLongtimeMaxBondLocal() == [fpl.getLongtimeMaxBond()]
    integ.run(20)
    assert fpl.getLongtimeMaxBond() >= longest
    fpl.resetLongtimeMaxBond()
    assert fpl.getLongtimeMaxBond() == 0.0
    fpl.remove()
    assert fpl.size() == 0 and fpl.getAllBonds() == []
    integ.run(5)
    assert fpl.getLongtimeMaxBond() == 0.0 and fene.computeEnergy() == 0.0
    ftl = espressopp.FixedTripleList(system.storage)
    ftl.addTriples([(0, 1, 2), (3, 4, 5)])
    assert ftl.size() == 2
    ftl.remove()
    assert ftl.size() == 0 and ftl.getTriples() == [[]]


def test_storage_remove_save_restore_and_arrays(on_oracle, capsys):
    """Storage (src/storage/Storage.py:198-535, Storage.cpp:315-358 and 804-869):
    removeParticle / removeAllParticles, savePositions / restorePositions /
    clearSavedPositions, printRealParticles and addParticlesArray."""
    system, integ = _fluid(n=512)
    st = system.storage
    lj = system.getInteraction(0)
    e_all = lj.computeEnergy()
    assert st.removeParticle(7) == 1 and st.removeParticle(7) == 0
    assert not st.particleExists(7) and st.getNRealParticles() == 511
    e_less = lj.computeEnergy()
    assert e_less != e_all
    integ.run(20)
    st.savePositions([3, 4, 999999])
    p3 = np.asarray(st.getParticle(3).pos)
    integ.run(20)
    assert not np.allclose(np.asarray(st.getParticle(3).pos), p3)
    st.restorePositions()
    assert np.array_equal(np.asarray(st.getParticle(3).pos), p3)
    st.clearSavedPositions()
    with pytest.raises(RuntimeError, match="nothing to restore"):
        st.restorePositions()
    st.printRealParticles()
    out = capsys.readouterr().out.splitlines()
    assert len(out) == 511 and out[0].startswith("CPU 0   ID 0     TYPE 0   POS(")
    st.removeAllParticles()
    assert st.getNRealParticles() == 0 and lj.computeEnergy() == 0.0
    arr = np.array([[10, 1.0, 1.0, 1.0, 0.1, 0.0, 0.0], [11, 2.2, 1.0, 1.0, 0.0, 0.0, 0.0]])
    st.addParticlesArray(arr, "id", "posx", "posy", "posz", "vx", "vy", "vz")
    assert st.getRealParticleIDs() == [10, 11]
    assert np.allclose(np.asarray(st.getParticle(10).v), [0.1, 0.0, 0.0])
    with pytest.raises(SyntaxError):
        st.addParticlesArray(arr, "id", "posx", "posy", "posz", "bogus", "vy", "vz")
    with pytest.raises(AssertionError):
        st.addParticlesArray(arr[:, :3], "id", "posx", "posy")


def test_capforce_setters(on_oracle):
    """CapForce (CapForce.cpp:38-102, 170-200): the constructor fixes absolute or
    per-component capping, setAbsCapForce / setCapForce change the value, the getters
    return it; the forces after a run obey the cap."""
    system, integ = _fluid(n=512)
    cap = espressopp.integrator.CapForce(system, 1.0e6)
    integ.addExtension(cap)
    cap.setAbsCapForce(0.5)
    assert cap.getAbsCapForce() == 0.5
    integ.run(0)
    f = system.storage.getAll()[3]
    assert np.max(np.sqrt(np.sum(f * f, axis=1))) <= 0.5 * (1 + 1e-12)
    system2, integ2 = _fluid(n=512)
    cap2 = espressopp.integrator.CapForce(system2, espressopp.Real3D(1e6, 1e6, 1e6))
    integ2.addExtension(cap2)
    cap2.setCapForce(espressopp.Real3D(0.1, 0.2, 0.3))
    assert tuple(cap2.getCapForce()) == (0.1, 0.2, 0.3)
    integ2.run(0)
    f2 = system2.storage.getAll()[3]
    assert np.all(np.abs(f2) <= np.array([0.1, 0.2, 0.3]) * (1 + 1e-12))
