"""The Python mirror on a decomposed storage: a reference-style script with
storage.DomainDecomposition(system, nodeGrid, cellGrid) and nodeGrid from
tools.decomp.nodeGrid(n) (slabs along z, espressopp_b200.domain) runs like the same script
with one node, the domains' systems driven through the FP64 oracle library: energies,
temperature, pressure, pair counts and trajectories agree; with two gloo ranks each rank
drives its own slab and gets the same results.
"""
import datetime
import math
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RC, SKIN = 2.5, 0.3


def _use_oracle():
    for p in (REPO, os.path.join(REPO, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from espressopp_b200 import _lib
    from simdriver import oracle_lib
    _lib._lib = oracle_lib()


def _script(nodes, bonds=False, steps=150):
    """A Lennard-Jones fluid (with a few FENE bonds) in the reference's script style;
    returns what the script reports."""
    import espressopp_b200 as espressopp
    x, y, z, Lx, Ly, Lz = espressopp.tools.lattice.createCubic(
        2197, 0.8442, perfect=False, RNG=espressopp.esutil.RNG(7))
    system = espressopp.System()
    system.rng = espressopp.esutil.RNG(5)
    system.bc = espressopp.bc.OrthorhombicBC(system.rng, (Lx, Ly, Lz))
    system.skin = SKIN
    ng = espressopp.tools.decomp.nodeGrid(nodes, (Lx, Ly, Lz), RC, SKIN)
    cg = espressopp.tools.decomp.cellGrid((Lx, Ly, Lz), ng, RC, SKIN)
    system.storage = espressopp.storage.DomainDecomposition(system, ng, cg)
    vel = espressopp.tools.velocities.gaussian(1.0, len(x), seed=3)
    system.storage.addParticles(
        [[k, espressopp.Real3D(x[k], y[k], z[k]), espressopp.Real3D(vel[0][k], vel[1][k],
                                                                    vel[2][k])]
         for k in range(len(x))], "id", "pos", "v")
    system.storage.decompose()
    vl = espressopp.VerletList(system, cutoff=RC)
    lj = espressopp.interaction.VerletListLennardJones(vl)
    lj.setPotential(0, 0, espressopp.interaction.LennardJones(1.0, 1.0, RC, "auto"))
    system.addInteraction(lj)
    fene = None
    if bonds:
        fpl = espressopp.FixedPairList(system.storage)
        fpl.addBonds([(k, k + 1) for k in range(0, 600, 2)])
        fene = espressopp.interaction.FixedPairListFENE(
            system, fpl, espressopp.interaction.FENE(K=30.0, r0=0.0, rMax=3.0))
        system.addInteraction(fene)
    integ = espressopp.integrator.VelocityVerlet(system)
    integ.dt = 0.005
    lang = espressopp.integrator.LangevinThermostat(system)
    lang.gamma = 1.0
    lang.temperature = 1.0
    integ.addExtension(lang)
    integ.run(steps)
    T = espressopp.analysis.Temperature(system).compute()
    P = espressopp.analysis.Pressure(system).compute()
    ids, pos, v, f, img = system.storage.getAll()
    return {"E": lj.computeEnergy(), "T": T, "P": P, "pairs": vl.totalSize(),
            "resorts": integ.getNumResorts(), "step": integ.step,
            "Eb": fene.computeEnergy() if fene else 0.0, "ids": ids,
            "pos": pos + img * np.array([Lx, Ly, Lz]), "nodes": tuple(
                system.storage.getNodeGrid())}


@pytest.mark.parametrize("nodes,bonds", [(2, False), (3, True)])
def test_decomposed_script_matches_one_node(nodes, bonds):
    _use_oracle()
    one = _script(1, bonds)
    dec = _script(nodes, bonds)
    assert dec["nodes"] == (1, 1, nodes) and one["nodes"] == (1, 1, 1)
    assert dec["pairs"] == one["pairs"] and dec["resorts"] == one["resorts"] > 0
    assert dec["step"] == one["step"] == 150
    for k in ("E", "T", "P", "Eb"):
        assert math.isclose(dec[k], one[k], rel_tol=1e-9, abs_tol=1e-12)
    assert np.array_equal(dec["ids"], one["ids"])
    assert np.max(np.abs(dec["pos"] - one["pos"])) < 1e-9


def test_decomposed_storage_refuses_whole_system_observables():
    _use_oracle()
    import espressopp_b200 as espressopp
    system = espressopp.System()
    system.rng = espressopp.esutil.RNG(5)
    system.bc = espressopp.bc.OrthorhombicBC(system.rng, (12.0, 12.0, 12.0))
    system.skin = SKIN
    system.storage = espressopp.storage.DomainDecomposition(system, (1, 1, 2), (4, 4, 2))
    system.storage.addParticles([[0, espressopp.Real3D(1, 1, 1)],
                                 [1, espressopp.Real3D(2, 2, 2)]], "id", "pos")
    system.storage.decompose()
    with pytest.raises(RuntimeError, match="decomposed"):
        espressopp.analysis.RadialDistrF(system).compute(10)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist
    _use_oracle()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import espressopp_b200 as espressopp
        assert espressopp.MPI.COMM_WORLD.size == world
        assert espressopp.MPI.COMM_WORLD.rank == rank
        res = _script(2, True, steps=100)
        np.save(os.path.join(out_dir, "pos%d.npy" % rank), res["pos"])
        with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
            f.write(repr({k: res[k] for k in ("E", "T", "P", "Eb", "pairs", "resorts")}))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_run_the_script(tmp_path):
    _use_oracle()
    ref = _script(2, True, steps=100)
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        got = eval((tmp_path / ("rank%d.txt" % r)).read_text())
        assert got["pairs"] == ref["pairs"] and got["resorts"] == ref["resorts"]
        for k in ("E", "T", "P", "Eb"):
            assert got[k] == ref[k]
        assert np.array_equal(np.load(tmp_path / ("pos%d.npy" % r)), ref["pos"])
