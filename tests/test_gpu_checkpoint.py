"""Checkpoint and resume through the Python mirror: the state of a Langevin LJ fluid
(positions, velocities, images from Storage.getAll), the integrator step and the RNG
state (RNG.saveState / loadState, src/esutil/RNG.cpp:86-138) are saved mid-run; a new
system built from them continues the trajectory of the uninterrupted run.  The Langevin
noise is counter-based (keyed on the seed and the particle id, counted by the step), so
the resumed noise is the same draw for draw."""
import numpy as np
import pytest

import espressopp_b200 as espressopp

pytestmark = pytest.mark.gpu


def _system(seed, particles=None):
    """A 1000-particle LJ fluid under Langevin (T 1, gamma 1, dt 0.005); `particles` =
    (ids, pos, v, img) restores a saved state instead of the lattice start."""
    x, y, z, Lx, Ly, Lz = espressopp.tools.lattice.createCubic(
        1000, 0.8442, perfect=False, RNG=espressopp.esutil.RNG(7))
    system = espressopp.System()
    system.rng = espressopp.esutil.RNG(seed)
    if particles is not None:
        system.rng.loadState("rng.checkpoint")
    system.bc = espressopp.bc.OrthorhombicBC(system.rng, (Lx, Ly, Lz))
    system.skin = 0.3
    cgrid = espressopp.tools.decomp.cellGrid((Lx, Ly, Lz), (1, 1, 1), 2.5, 0.3)
    system.storage = espressopp.storage.DomainDecomposition(system, (1, 1, 1), cgrid)
    if particles is None:
        system.storage.addParticles([[k, espressopp.Real3D(x[k], y[k], z[k])]
                                     for k in range(len(x))], "id", "pos")
    else:
        ids, pos, vel, img = particles
        system.storage.addParticles([[int(ids[k]), espressopp.Real3D(pos[k]),
                                      espressopp.Real3D(vel[k])] for k in range(len(ids))],
                                    "id", "pos", "v")
        system.storage.setImages(ids, img)
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


def test_checkpoint_resume_continues_the_trajectory(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    full, integ_full = _system(2024)
    integ_full.run(300)
    integ_full.run(200)
    part, integ_part = _system(2024)
    integ_part.run(300)
    ids, pos, vel, _, img = part.storage.getAll()
    assert np.any(img != 0)  # particles have crossed the box
    # positions are folded only at re-sorts, so some lie just outside the box; addParticles
    # folds them again, so save them folded (OrthorhombicBC::foldCoordinate arithmetic)
    L = np.asarray(part.bc.boxL)
    t = np.floor(pos * (1.0 / L))
    pos, img = pos - t * L, img + t.astype(np.int32)
    part.rng.saveState(integ_part.step)
    (tmp_path / "rng.checkpoint").write_text((tmp_path / "rng.300").read_text())
    # the resumed system starts from another seed; loadState brings back the saved one
    resumed, integ_res = _system(1, (ids, pos, vel, img))
    assert resumed.rng.get_seed() == 2024
    integ_res.step = integ_part.step
    integ_res.run(200)
    assert integ_res.step == integ_full.step == 500
    a = full.storage.getAll()
    b = resumed.storage.getAll()
    assert np.array_equal(a[0], b[0])
    unf = lambda s: s[1] + s[4] * np.asarray(full.bc.boxL)
    assert np.max(np.abs(unf(a) - unf(b))) < 1e-8
    assert np.max(np.abs(a[2] - b[2])) < 1e-7
    # and it differs from a resume without the step (the noise is counted by the step)
    other, integ_o = _system(1, (ids, pos, vel, img))
    integ_o.run(200)
    assert np.max(np.abs(unf(other.storage.getAll()) - unf(a))) > 1e-3


def test_modify_particle_pos_resets_the_image():
    """modifyParticle(pid, 'pos', ...) takes the position as unfolded and zeroes the
    image; 'img' sets it (Storage.py:374-400)."""
    system, integ = _system(5)
    st = system.storage
    st.modifyParticle(3, "img", (2, -1, 4))
    assert tuple(st.getAll()[4][3]) == (2, -1, 4)
    st.modifyParticle(3, "pos", (1.0, 2.0, 3.0))
    ids, pos, _, _, img = st.getAll()
    assert tuple(img[3]) == (0, 0, 0) and tuple(pos[3]) == (1.0, 2.0, 3.0)
    integ.run(1)
