"""Spatial domain decomposition on the GPU: two and three slab domains, each a system of
the CUDA library, driven in one process on one device (the halo refresh and the
migration go through the host, so no kernel waits on another domain).  Against one
undecomposed CUDA system and against the FP64 oracle: the pair set (bit-exact), energies,
virials, kinetic sums and forces, and a Langevin run with the same re-sort steps
(DomainDecomposition.cpp:1031-1391, VelocityVerlet.cpp:63-169).
"""
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from espressopp_b200.domain import SpatialDecomposition
from simdriver import Sim, cell_grid, cuda_lib, lattice, mb_velocities, oracle_lib

pytestmark = pytest.mark.gpu

RC, SKIN = 2.5, 0.3
SHIFT = 4.0 * (RC ** -12 - RC ** -6)


def _inputs(n_side):
    pos, box = lattice(n_side, 0.8442, 0.05, 3)
    vel = mb_velocities(len(pos), 1.0, 4)
    return np.arange(len(pos), dtype=np.int64), pos, vel, box


def _plain(lib, prec, ids, pos, vel, box, cg):
    s = Sim(lib, box, SKIN, cg, precision=prec, seed=4)
    s.add(ids, pos, vel)
    s.decompose()
    s.vl(RC)
    s.lj(0, 0, 1.0, 1.0, RC, SHIFT)
    s.integrator(0.005)
    s.langevin(1.0, 1.0)
    return s


def _decomposed(prec, ids, pos, vel, box, cg, D, exchange="host"):
    dd = SpatialDecomposition(box, SKIN, cg, D, precision=prec, seed=4, lib=cuda_lib(),
                              exchange=exchange)
    dd.add_particles(ids, pos, vel)
    dd.decompose()
    dd.vl_create(RC)
    dd.lj_set(0, 0, 1.0, 1.0, RC, SHIFT)
    dd.integrator_set(0.005)
    dd.langevin_set(1, 1.0, 1.0)
    return dd


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_decomposed_fluid_matches_one_system(D, prec):
    ids, pos, vel, box = _inputs(16)  # 4096 particles, 5^3 cells
    cg = cell_grid(box, RC, SKIN)
    one = _plain(cuda_lib(), prec, ids, pos, vel, box, cg)
    orc = _plain(oracle_lib(), _abi.PREC_FP64, ids, pos, vel, box, cg)
    dd = _decomposed(prec, ids, pos, vel, box, cg, D)
    assert all(h > 0 for _, h in dd.domain_sizes())
    for s in (one, orc, dd):
        s.run(0)
    assert dd.vl_size() == orc.vl_size()
    assert np.array_equal(dd.vl_pairs(), orc.pairs())
    assert dd.vl_digest() == orc.digest() == one.digest()
    fp64 = prec == _abi.PREC_FP64
    assert math.isclose(dd.energy(_abi.IA_LJ), orc.energy(_abi.IA_LJ), rel_tol=1e-10)
    assert math.isclose(dd.virial(_abi.IA_LJ), orc.virial(_abi.IA_LJ), rel_tol=1e-10)
    k, n = dd.kinetic()
    assert n == len(ids) and math.isclose(k, orc.kinetic()[0], rel_tol=1e-12)
    f, fo = dd.get_particles(ids)[2], orc.particles(ids)[2]
    assert math.sqrt(np.sum((f - fo) ** 2) / np.sum(fo ** 2)) < (1e-12 if fp64 else 1e-5)
    # against the undecomposed CUDA system: the same kernels on lists in another order
    # (mixed precision: FP32 sums in that order)
    f1 = one.particles(ids)[2]
    assert math.sqrt(np.sum((f - f1) ** 2) / np.sum(f1 ** 2)) < (1e-12 if fp64 else 1e-6)
    for s in (one, dd):
        s.run(120)
    assert dd.resorts == one.num_resorts() > 3
    x, _, _, img = dd.get_particles(ids)
    x1, _, _, i1 = one.particles(ids)
    if fp64:
        assert np.array_equal(img, i1) and np.max(np.abs(x - x1)) < 1e-9
        assert dd.vl_digest() == one.digest()
    else:  # the FP32 rounding differences grow along the run
        assert np.max(np.abs((x + img * box) - (x1 + i1 * box))) < 1e-3


def test_decomposed_melt_bonds_on_gpu():
    """Kremer-Grest melt over 3 slabs (FP64): FENE bonds across slab boundaries, capped
    WCA, Langevin; energies and positions against one CUDA system, and the long-time
    maximum bond."""
    from espressopp_b200.tools import topology
    pos, bonds, L = topology.polymer_melt(20, 50, 0.85, seed=3)
    box = np.array([L, L, L])
    rc = 2.0 ** (1.0 / 6.0)
    shift = 4.0 * ((1.0 / rc ** 2) ** 6 - (1.0 / rc ** 2) ** 3)
    ids = np.arange(1, len(pos) + 1, dtype=np.int64)
    cg = cell_grid(box, rc, 0.3)
    one = Sim(cuda_lib(), box, 0.3, cg, seed=11)
    one.add(ids, pos)
    one.decompose()
    one.vl(rc)
    one.lj(0, 0, 1.0, 1.0, rc, shift, caprad=0.9)
    one.bonds(bonds)
    one.fene(30.0, 0.0, 1.5)
    one.integrator(0.01)
    one.langevin(0.5, 1.0)
    dd = SpatialDecomposition(box, 0.3, cg, 3, seed=11, lib=cuda_lib())
    dd.add_particles(ids, pos)
    dd.decompose()
    dd.vl_create(rc)
    dd.lj_set(0, 0, 1.0, 1.0, rc, shift, caprad=0.9)
    dd.bonds_add(bonds)
    dd.fene_set(30.0, 0.0, 1.5)
    dd.integrator_set(0.01)
    dd.langevin_set(1, 0.5, 1.0)
    for s in (one, dd):
        s.run(100)
    assert dd.resorts == one.num_resorts() > 0
    for which in (_abi.IA_LJ, _abi.IA_FENE):
        assert math.isclose(dd.energy(which), one.energy(which), rel_tol=1e-9)
    x, _, _, img = dd.get_particles(ids)
    x1, _, _, i1 = one.particles(ids)
    assert np.max(np.abs(x - x1)) < 1e-8 and np.array_equal(img, i1)
    m1 = np.zeros(1)
    _abi.call(one.lib, "espp_bonds_max_sqr", one.h, _abi.dptr(m1))
    assert math.isclose(dd.bonds_max_sqr(), m1[0], rel_tol=1e-12)


def test_storage_removal_matches_the_oracle():
    """storage.removeParticle / removeAllParticles of the Python mirror replace the
    particle set through espp_dd_load (state kept, no halo copies): energies before and
    after a run against the oracle driven the same way."""
    import espressopp_b200 as espressopp
    from espressopp_b200 import _lib
    saved = _lib._lib
    out = []
    try:
        for lib in (oracle_lib(), cuda_lib()):
            _lib._lib = lib
            x, y, z, Lx, Ly, Lz = espressopp.tools.lattice.createCubic(
                1000, 0.8442, perfect=False, RNG=espressopp.esutil.RNG(5))
            system = espressopp.System()
            system.rng = espressopp.esutil.RNG(6)
            system.bc = espressopp.bc.OrthorhombicBC(system.rng, (Lx, Ly, Lz))
            system.skin = SKIN
            cg = espressopp.tools.decomp.cellGrid((Lx, Ly, Lz), (1, 1, 1), RC, SKIN)
            system.storage = espressopp.storage.DomainDecomposition(system, (1, 1, 1), cg)
            system.storage.addParticles([[k, espressopp.Real3D(x[k], y[k], z[k])]
                                         for k in range(len(x))], "id", "pos")
            system.storage.decompose()
            vl = espressopp.VerletList(system, cutoff=RC)
            lj = espressopp.interaction.VerletListLennardJones(vl)
            lj.setPotential(0, 0, espressopp.interaction.LennardJones(1.0, 1.0, RC, "auto"))
            system.addInteraction(lj)
            integ = espressopp.integrator.VelocityVerlet(system)
            integ.dt = 0.005
            integ.run(10)
            for pid in (0, 17, 500):
                system.storage.removeParticle(pid)
            e1 = lj.computeEnergy()
            integ.run(20)
            ids, pos = system.storage.getAll()[:2]
            out.append((e1, lj.computeEnergy(), ids, pos, vl.totalSize()))
            system.storage.removeAllParticles()
            assert lj.computeEnergy() == 0.0
    finally:
        _lib._lib = saved
    (o1, o2, oi, op, on), (g1, g2, gi, gp, gn) = out
    assert np.array_equal(oi, gi) and len(gi) == 997 and on == gn
    assert math.isclose(g1, o1, rel_tol=1e-10) and math.isclose(g2, o2, rel_tol=1e-9)
    assert np.max(np.abs(gp - op)) < 1e-9


def test_mirror_script_with_two_nodes_on_gpu():
    """A reference-style script with nodeGrid (1, 1, 2) (two slab systems on one device)
    against the same script with one node, both on the CUDA library (FP64): energy,
    temperature, pressure, pair count, re-sorts and trajectory."""
    import sys as _sys
    import os as _os
    _sys.path.insert(0, _os.path.dirname(_os.path.abspath(__file__)))
    import test_domain_mirror_cpu as m
    from espressopp_b200 import _lib
    saved = _lib._lib
    _lib._lib = cuda_lib()
    try:
        one = m._script(1, True)
        dec = m._script(2, True)
    finally:
        _lib._lib = saved
    assert dec["pairs"] == one["pairs"] and dec["resorts"] == one["resorts"] > 0
    for k in ("E", "T", "P", "Eb"):
        assert math.isclose(dec[k], one[k], rel_tol=1e-9, abs_tol=1e-12)
    assert np.max(np.abs(dec["pos"] - one["pos"])) < 1e-9


def test_direct_halo_exchange_on_gpu():
    """The halo refresh in device buffers (espp_dd_read_positions / espp_dd_write_halo,
    device-to-device, no host copies) gives the host-array refresh's trajectory bit for
    bit (3 domains on one device, FP64 and mixed)."""
    ids, pos, vel, box = _inputs(16)
    cg = cell_grid(box, RC, SKIN)
    for prec in (_abi.PREC_FP64, _abi.PREC_MIXED):
        out = []
        for exchange in ("host", "direct"):
            dd = _decomposed(prec, ids, pos, vel, box, cg, 3, exchange)
            dd.run(100)
            out.append((dd.get_particles(ids), dd.resorts, dd.vl_digest()))
            dd.close()
        (a, ra, ga), (b, rb, gb) = out
        assert ra == rb > 0 and ga == gb
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
