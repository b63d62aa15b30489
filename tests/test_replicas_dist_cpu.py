"""Parallel tempering with the replicas shared out among ranks, on CPU: two gloo ranks
(world size 2) driving the FP64 oracle library, which exports the same C ABI as the
CUDA library.  Each rank steps only its own replicas; exchange() gathers (E_pot, T, N)
of all replicas with one all-reduce and applies the Metropolis rule of
ParallelTempering.exchange (src/ParallelTempering.py:164-203) on every rank.  The
exchange decisions and the temperatures must be those of the same run in one process.
"""
import datetime
import os
import random
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SIDES = [5, 6, 4, 7, 5, 6]  # replica lattices: 125 .. 343 particles
ROUNDS = 4


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _use_oracle():
    for p in (REPO, os.path.join(REPO, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from espressopp_b200 import _lib
    from simdriver import oracle_lib
    _lib._lib = oracle_lib()


def _build(pt, n, side):
    import espressopp_b200 as espressopp
    x, y, z, Lx, Ly, Lz = espressopp.tools.lattice.createCubic(
        side ** 3, 0.8442, perfect=False, RNG=espressopp.esutil.RNG(11 + n))
    system = espressopp.System()
    system.rng = espressopp.esutil.RNG(100 + n)
    system.bc = espressopp.bc.OrthorhombicBC(system.rng, (Lx, Ly, Lz))
    system.skin = 0.3
    cg = espressopp.tools.decomp.cellGrid((Lx, Ly, Lz), (1, 1, 1), 1.5, 0.3)
    system.storage = espressopp.storage.DomainDecomposition(system, (1, 1, 1), cg)
    system.storage.addParticles([[k, espressopp.Real3D(x[k], y[k], z[k])]
                                 for k in range(len(x))], "id", "pos")
    system.storage.decompose()
    vl = espressopp.VerletList(system, cutoff=1.5)
    lj = espressopp.interaction.VerletListLennardJones(vl)
    lj.setPotential(0, 0, espressopp.interaction.LennardJones(1.0, 1.0, 1.5, "auto"))
    system.addInteraction(lj)
    integ = espressopp.integrator.VelocityVerlet(system)
    integ.dt = 0.005
    lang = espressopp.integrator.LangevinThermostat(system)
    lang.gamma = 1.0
    lang.temperature = 0.7 * (2.0 / 0.7) ** (n / (len(SIDES) - 1))
    integ.addExtension(lang)
    pt.setIntegrator(integ, lang)
    pt.setAnalysisE(lj)
    pt.setAnalysisT(espressopp.analysis.Temperature(system))
    pt.setAnalysisNPart(espressopp.analysis.NPart(system))


def _run(group):
    """The exchange decisions of every round and the thermostat temperatures of this
    process's replicas {replica: T}."""
    import espressopp_b200 as espressopp
    pt = espressopp.ParallelTempering(NumberOfSystems=len(SIDES), RNG=random.Random(335977),
                                      group=group, sizes=[s ** 3 for s in SIDES])
    for n, side in enumerate(SIDES):
        if pt.startDefiningSystem(n):
            _build(pt, n, side)
        pt.endDefiningSystem(n)
    rounds = []
    for _ in range(ROUNDS):
        pt.run(30)
        rounds.append([(m, n, round(d, 12), bool(ok)) for m, n, d, _, ok in pt.exchange()])
    temps = {n: pt._thermo[n].temperature for n in pt._local}
    return rounds, temps, pt._local


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist
    _use_oracle()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        rounds, temps, local = _run(dist.group.WORLD)
        with open(os.path.join(out_dir, "rank%d" % rank), "w") as f:
            f.write(repr((rounds, temps, local)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_partition_balances_particles():
    sys.path.insert(0, REPO)
    from espressopp_b200.parallel_tempering import partition_replicas
    rng = np.random.Generator(np.random.PCG64(4))
    sizes = rng.integers(2000, 64001, size=64)
    for world in (1, 2, 4, 8):
        owner = partition_replicas(sizes, world)
        load = [int(sum(s for s, o in zip(sizes, owner) if o == r)) for r in range(world)]
        assert sorted(set(owner)) == list(range(world))
        assert max(load) - min(load) <= max(sizes)
        assert owner == partition_replicas(list(sizes), world)


def test_sharded_exchange_matches_one_process(tmp_path):
    _use_oracle()
    ref_rounds, ref_temps, ref_local = _run(None)
    assert ref_local == list(range(len(SIDES)))
    assert any(ok for r in ref_rounds for *_, ok in r)  # some swaps are accepted
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    owned = []
    for r in range(2):
        rounds, temps, local = eval((tmp_path / ("rank%d" % r)).read_text())
        assert rounds == ref_rounds
        assert local and all(temps[n] == ref_temps[n] for n in local)
        owned += local
    assert sorted(owned) == list(range(len(SIDES)))
