"""standard_system.Default / Minimal / LennardJones / PolymerMelt
(src/standard_system/Default.py, Minimal.py:50-86, LennardJones.py:1-145,
PolymerMelt.py:62-175)."""
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


def Minimal(num_particles, box, rc=1.12246, skin=0.3, dt=0.005, temperature=None,
            precision=None):
    """A system of num_particles at random positions in the box, at rest, with no
    interactions (Minimal.py:50-86); ids 1..num_particles, type 0, mass 1."""
    system, integ = Default(box, rc, skin, dt, temperature, precision=precision)
    props = ["id", "type", "mass", "pos", "v"]
    parts = [[pid, 0, 1.0, system.bc.getRandomPos(), core.Real3D(0.0, 0.0, 0.0)]
             for pid in range(1, num_particles + 1)]
    system.storage.addParticles(parts, *props)
    system.storage.decompose()
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


def PolymerMelt(num_chains, monomers_per_chain, box=(0, 0, 0), bondlen=0.97, rc=1.12246,
                skin=0.3, dt=0.005, epsilon=1.0, sigma=1.0, shift="auto", temperature=None,
                xyzfilename=None, xyzrfilename=None, precision=None):
    """Random-walk polymer melt with LJ (type 0 pairs) and FENE(K=30, r0=0, rMax=1.5)
    bonds (PolymerMelt.py:62-175).  Chains are grown with tools.topology.polymerRW from
    random start positions.  Every bead gets type 0: the reference numbers the chains'
    types 0, 1, 2, ... while setting the LJ potential for types (0, 0) only, which leaves
    all chains but the first without pair interactions."""
    from .tools import topology
    if xyzrfilename:
        raise ValueError("xyzr input is not supported; use xyzfilename")
    if xyzfilename:
        pidf, typef, xf, yf, zf, vxf, vyf, vzf, Lx, Ly, Lz = readxyz(xyzfilename)
        box = (Lx, Ly, Lz)
    elif box[0] <= 0 or box[1] <= 0 or box[2] <= 0:
        box = (100, 100, 100)
    system, integ = Default(box, rc, skin, dt, temperature, precision=precision)
    props = ["id", "type", "mass", "pos", "v"]
    bondlist = core.FixedPairList(system.storage)
    pid = 1
    for i in range(num_chains):
        chain = []
        if xyzfilename:
            bonds = []
            for k in range(monomers_per_chain):
                idx = i * monomers_per_chain + k
                chain.append([pidf[idx], typef[idx], 1.0, core.Real3D(xf[idx], yf[idx], zf[idx]),
                              core.Real3D(vxf[idx], vyf[idx], vzf[idx])])
                if k > 0:
                    bonds.append((pidf[idx - 1], pidf[idx]))
        else:
            startpos = system.bc.getRandomPos()
            positions, bonds = topology.polymerRW(pid, startpos, monomers_per_chain, bondlen)
            for k in range(monomers_per_chain):
                chain.append([pid + k, 0, 1.0, positions[k], core.Real3D(0.0)])
            pid += monomers_per_chain
        system.storage.addParticles(chain, *props)
        bondlist.addBonds(bonds)
    system.storage.decompose()
    vl = core.VerletList(system, cutoff=rc)
    ia = interaction.VerletListLennardJones(vl)
    ia.setPotential(0, 0, interaction.LennardJones(epsilon, sigma, rc, shift))
    system.addInteraction(ia)
    fene = interaction.FixedPairListFENE(system, bondlist,
                                         interaction.FENE(K=30.0, r0=0.0, rMax=1.5))
    system.addInteraction(fene)
    return system, integ
