"""standard_system.Default / LennardJones (src/standard_system/Default.py,
LennardJones.py:1-145)."""
from . import core, integrator as _integrator, interaction, storage as _storage
from .tools import decomp
from .tools.DumpConfigurations import readxyz


def Default(box, rc=1.12246, skin=0.3, dt=0.005, temperature=None, halfCellInt=1,
            precision=None):
    system = core.System()
    system.rng = core.RNG()
    system.bc = core.OrthorhombicBC(system.rng, box)
    system.skin = skin
    nodeGrid = decomp.nodeGrid(1, box, rc, skin)
    cellGrid = decomp.cellGrid(box, nodeGrid, rc, skin, halfCellInt)
    system.storage = _storage.DomainDecomposition(system, nodeGrid, cellGrid, halfCellInt,
                                                  precision=precision)
    integ = _integrator.VelocityVerlet(system)
    integ.dt = dt
    if temperature is not None:
        t = _integrator.LangevinThermostat(system)
        t.gamma = 1.0
        t.temperature = temperature
        integ.addExtension(t)
    return system, integ


def LennardJones(num_particles, box=(0, 0, 0), rc=1.12246, skin=0.3, dt=0.005, epsilon=1.0,
                 sigma=1.0, shift="auto", temperature=None, xyzfilename=None,
                 xyzrfilename=None, precision=None):
    if xyzfilename:
        pid, typ, x, y, z, vx, vy, vz, Lx, Ly, Lz = readxyz(xyzfilename)
        box = (Lx, Ly, Lz)
        num_particles = len(pid)
    system, integ = Default(box, rc, skin, dt, temperature, precision=precision)
    props = ["id", "type", "mass", "pos", "v"]
    parts = []
    if xyzfilename:
        for k in range(num_particles):
            parts.append([pid[k], typ[k], 1.0, core.Real3D(x[k], y[k], z[k]),
                          core.Real3D(vx[k], vy[k], vz[k])])
    else:
        for p in range(1, num_particles + 1):
            parts.append([p, 0, 1.0, system.bc.getRandomPos(), core.Real3D(0.0)])
    system.storage.addParticles(parts, *props)
    system.storage.decompose()
    vl = core.VerletList(system, cutoff=rc)
    pot = interaction.LennardJones(epsilon, sigma, rc, shift)
    ia = interaction.VerletListLennardJones(vl)
    ia.setPotential(0, 0, pot)
    system.addInteraction(ia)
    return system, integ
