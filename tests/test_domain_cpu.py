"""Spatial domain decomposition (espressopp_b200.domain) on CPU, the domains' systems
driven through the FP64 oracle library (the same C ABI as the CUDA library).

The decomposition follows DomainDecomposition over several ranks (src/storage/
DomainDecomposition.cpp:1031-1158 migration, :1243-1391 ghost frames) with slabs of whole
cells along z: against one undecomposed system the pair set, energies, virials, kinetic
sums and forces must agree, and a Langevin run must re-sort on the same steps and follow
the same trajectory (summation order aside).  The same holds with the domains shared out
among two gloo ranks (world size 2).
"""
import ctypes
import datetime
import math
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from espressopp_b200 import _abi
from espressopp_b200.domain import SpatialDecomposition, fold_cells, slab_bounds
from simdriver import Sim, cell_grid, lattice, mb_velocities, oracle_lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RC, SKIN = 2.5, 0.3
SHIFT = 4.0 * (RC ** -12 - RC ** -6)


def _fluid_inputs(n_side=10):
    pos, box = lattice(n_side, 0.8442, 0.05, 3)
    vel = mb_velocities(len(pos), 1.0, 4)
    return np.arange(len(pos), dtype=np.int64), pos, vel, box


def _plain(ids, pos, vel, box, cg, h=1):
    s = Sim(oracle_lib(), box, SKIN, cg, seed=4, half_cell_int=h)
    s.add(ids, pos, vel)
    s.decompose()
    s.vl(RC)
    s.lj(0, 0, 1.0, 1.0, RC, SHIFT)
    s.integrator(0.005)
    s.langevin(1.0, 1.0)
    return s


def _decomposed(ids, pos, vel, box, cg, D, comm=None, h=1, exchange="host"):
    dd = SpatialDecomposition(box, SKIN, cg, D, lib=oracle_lib(), seed=4, comm=comm,
                              half_cell_int=h, exchange=exchange)
    dd.add_particles(ids, pos, vel)
    dd.decompose()
    dd.vl_create(RC)
    dd.lj_set(0, 0, 1.0, 1.0, RC, SHIFT)
    dd.integrator_set(0.005)
    dd.langevin_set(1, 1.0, 1.0)
    return dd


def test_host_fold_matches_the_library():
    """The host's fold and cell map (which decides ownership) gives the library's folded
    positions and images bit for bit, also for positions outside the box."""
    rng = np.random.Generator(np.random.PCG64(8))
    box = np.array([10.3, 11.7, 12.9])
    cg = [3, 4, 4]
    pos = rng.uniform(-25.0, 40.0, size=(500, 3))
    pos[:6] = [[0.0, 0.0, 0.0], box, box * (1 - 1e-16), [-1e-17, 5, 5], [10.3, 11.7, -12.9],
               [2 * 10.3, 0.5, 3 * 12.9]]
    ids = np.arange(len(pos), dtype=np.int64)
    s = Sim(oracle_lib(), box, SKIN, cg)
    s.add(ids, pos)
    s.decompose()
    got, _, _, img = s.particles(ids)
    for k in range(3):
        x1, t1, _ = fold_cells(pos[:, k], box[k], cg[k])  # espp_add_particles
        x2, t2, c2 = fold_cells(x1, box[k], cg[k])        # the re-sort
        assert np.array_equal(x2, got[:, k])
        assert np.array_equal(t1 + t2, img[:, k])
        assert c2.min() >= 0 and c2.max() < cg[k]


def test_slabs_and_halo_layers():
    assert slab_bounds(7, 3) == [(0, 2), (2, 4), (4, 7)]
    _, _, _, box = _fluid_inputs(6)
    cg = [4, 4, 6]
    dd = SpatialDecomposition(box, SKIN, cg, 3, lib=oracle_lib(), half_cell_int=1)
    assert [list(np.nonzero(dd.halo_of[e])[0]) for e in range(3)] == [[2, 5], [1, 4], [0, 3]]
    dd = SpatialDecomposition(box, SKIN, cg, 2, lib=oracle_lib())
    assert [list(np.nonzero(dd.halo_of[e])[0]) for e in range(2)] == [[3, 5], [0, 2]]
    dd = SpatialDecomposition(box, SKIN, cg, 1, lib=oracle_lib())
    assert not dd.halo_of.any()
    with pytest.raises(ValueError):
        SpatialDecomposition(box, SKIN, cg, 7, lib=oracle_lib())


@pytest.mark.parametrize("D", [1, 2, 3])
def test_decomposed_fluid_matches_one_system(D):
    ids, pos, vel, box = _fluid_inputs(10)
    cg = cell_grid(box, RC, SKIN)
    ref = _plain(ids, pos, vel, box, cg)
    dd = _decomposed(ids, pos, vel, box, cg, D)
    sizes = dd.domain_sizes()
    assert sum(o for o, _ in sizes) == len(ids)
    assert (D == 1) == all(h == 0 for _, h in sizes)
    for s in (ref, dd):
        s.run(0)
    assert dd.vl_size() == ref.vl_size()
    assert np.array_equal(dd.vl_pairs(), ref.pairs())
    assert dd.vl_digest() == ref.digest()
    assert math.isclose(dd.energy(_abi.IA_LJ), ref.energy(_abi.IA_LJ), rel_tol=1e-12)
    assert math.isclose(dd.virial(_abi.IA_LJ), ref.virial(_abi.IA_LJ), rel_tol=1e-12)
    assert np.allclose(dd.virial_tensor(_abi.IA_LJ), ref.virial_tensor(_abi.IA_LJ),
                       rtol=1e-12, atol=1e-9)
    k, n = dd.kinetic()
    assert n == len(ids) and math.isclose(k, ref.kinetic()[0], rel_tol=1e-13)
    f = dd.get_particles(ids)[2]
    assert np.max(np.abs(f - ref.particles(ids)[2])) < 1e-10
    ref.run(200)
    dd.run(200)
    assert dd.resorts == ref.num_resorts() > 5
    x, v, _, img = dd.get_particles(ids)
    xr, vr, _, ir = ref.particles(ids)
    assert np.max(np.abs(x - xr)) < 1e-9 and np.max(np.abs(v - vr)) < 1e-8
    assert np.array_equal(img, ir)
    assert np.array_equal(dd.vl_pairs(), ref.pairs())
    assert math.isclose(dd.energy(_abi.IA_LJ), ref.energy(_abi.IA_LJ), rel_tol=1e-10)


def test_decomposed_melt_with_bonds_and_half_cells():
    """A Kremer-Grest melt (WCA + FENE, capped LJ, Langevin) over 3 slabs at halfCellInt
    2: bonds crossing slab boundaries are computed by both owners from halo copies and
    counted once; the long-time maximum bond is the system's."""
    from espressopp_b200.tools import topology
    pos, bonds, L = topology.polymer_melt(12, 30, 0.85, seed=5)
    box = np.array([L, L, L])
    rc = 2.0 ** (1.0 / 6.0)
    shift = 4.0 * ((1.0 / rc ** 2) ** 6 - (1.0 / rc ** 2) ** 3)
    ids = np.arange(1, len(pos) + 1, dtype=np.int64)
    h = 2
    cg = cell_grid(box, rc, 0.3, h)
    ref = Sim(oracle_lib(), box, 0.3, cg, seed=7, half_cell_int=h)
    ref.add(ids, pos)
    ref.decompose()
    ref.vl(rc)
    ref.lj(0, 0, 1.0, 1.0, rc, shift, caprad=0.9)
    ref.bonds(bonds)
    ref.fene(30.0, 0.0, 1.5)
    ref.integrator(0.01)
    ref.langevin(0.5, 1.0)
    dd = SpatialDecomposition(box, 0.3, cg, 3, lib=oracle_lib(), seed=7, half_cell_int=h)
    dd.add_particles(ids, pos)
    dd.decompose()
    dd.vl_create(rc)
    dd.lj_set(0, 0, 1.0, 1.0, rc, shift, caprad=0.9)
    dd.bonds_add(bonds)
    dd.fene_set(30.0, 0.0, 1.5)
    dd.integrator_set(0.01)
    dd.langevin_set(1, 0.5, 1.0)
    for s in (ref, dd):
        s.run(60)
    assert dd.resorts == ref.num_resorts() > 0
    for which in (_abi.IA_LJ, _abi.IA_FENE):
        assert math.isclose(dd.energy(which), ref.energy(which), rel_tol=1e-9)
    x, _, _, img = dd.get_particles(ids)
    xr, _, _, ir = ref.particles(ids)
    assert np.max(np.abs(x - xr)) < 1e-8 and np.array_equal(img, ir)
    mref = np.zeros(1)
    _abi.call(ref.lib, "espp_bonds_max_sqr", ref.h, _abi.dptr(mref))
    assert math.isclose(dd.bonds_max_sqr(), mref[0], rel_tol=1e-9)


def test_decomposition_refuses_what_needs_the_whole_system():
    ids, pos, vel, box = _fluid_inputs(6)
    cg = cell_grid(box, 1.5, SKIN)
    dd = SpatialDecomposition(box, SKIN, cg, 2, lib=oracle_lib())
    dd.add_particles(ids, pos, vel)
    dd.decompose()
    dd.vl_create(1.5)
    dd.integrator_set(0.005)
    t = np.array([0, 1, 2], np.int64)
    _abi.call(dd.lib, "espp_triples_add", dd.handles[dd.local[0]], 1, _abi.i64ptr(t))
    with pytest.raises(RuntimeError, match="not available with halo"):
        dd.run(1)
    with pytest.raises(RuntimeError, match="not available with halo"):
        dd.energy(_abi.IA_COSINE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir, D, exchange):
    import torch.distributed as dist
    for p in (REPO, os.path.join(REPO, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from espressopp_b200.domain import TorchComm
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        ids, pos, vel, box = _fluid_inputs(13)
        dd = _decomposed(ids, pos, vel, box, cell_grid(box, RC, SKIN), D, comm=TorchComm(dist),
                         exchange=exchange)
        dd.run(150)
        x, v, _, img = dd.get_particles(ids)
        out = (dd.local, dd.resorts, dd.vl_digest(), dd.energy(_abi.IA_LJ), dd.kinetic())
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), x=x, v=v, img=img)
        with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
            f.write(repr(out))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("D,exchange", [(2, "host"), (4, "host"), (4, "direct")])
def test_two_gloo_ranks_match_one_process(tmp_path, D, exchange):
    """Also with the halo positions sent point to point in library-space buffers
    (exchange 'direct': gloo isend/irecv of CPU tensors for the oracle)."""
    ids, pos, vel, box = _fluid_inputs(13)  # 4 cells along z
    cg = cell_grid(box, RC, SKIN)
    ref = _decomposed(ids, pos, vel, box, cg, D)
    ref.run(150)
    xr, vr, _, ir = ref.get_particles(ids)
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path), D, exchange), nprocs=2,
                       join=True, start_method="spawn")
    held = []
    for r in range(2):
        local, resorts, digest, e, kin = eval((tmp_path / ("rank%d.txt" % r)).read_text())
        z = np.load(tmp_path / ("rank%d.npz" % r))
        assert resorts == ref.resorts and digest == ref.vl_digest()
        assert math.isclose(e, ref.energy(_abi.IA_LJ), rel_tol=1e-12)
        assert kin[1] == len(ids) and math.isclose(kin[0], ref.kinetic()[0], rel_tol=1e-12)
        assert np.array_equal(z["x"], xr) and np.array_equal(z["v"], vr)
        assert np.array_equal(z["img"], ir)
        held += local
    assert sorted(held) == list(range(D))


def test_direct_halo_exchange_in_one_process():
    """The halo refresh through library-space buffers gives the host-array refresh's
    trajectory bit for bit (3 domains in one process)."""
    ids, pos, vel, box = _fluid_inputs(10)
    cg = cell_grid(box, RC, SKIN)
    out = []
    for exchange in ("host", "direct"):
        dd = _decomposed(ids, pos, vel, box, cg, 3, exchange=exchange)
        dd.run(120)
        out.append((dd.get_particles(ids), dd.resorts, dd.vl_digest()))
    (a, ra, ga), (b, rb, gb) = out
    assert ra == rb > 0 and ga == gb
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_decomposed_melt_with_tables_exclusions_and_caps(tmp_path):
    """Tabulated pair and bond potentials (Akima tables of the reference's tabulated
    test), Verlet-list exclusions of the bonded pairs, Langevin exclusions and a
    per-component CapForce on a melt over 3 slabs: energies of both tables, pair set,
    re-sorts and trajectory equal one system's (oracle)."""
    from espressopp_b200.tools import topology
    from simdriver import polymer_tab_tables
    tl, tf, _, _ = polymer_tab_tables(tmp_path, oracle_lib())
    pos, bonds, L = topology.polymer_melt(12, 30, 0.85, seed=8)
    box = np.array([L, L, L])
    ids = np.arange(1, len(pos) + 1, dtype=np.int64)
    cg = cell_grid(box, 1.12, 0.3)
    excl = np.asarray(bonds, np.int64)
    lexcl = ids[::7]
    cap = np.array([50.0, 60.0, 70.0])

    def setup(s, dd):
        if dd:
            s.vl_create(1.12, excl)
            s.tab_pair_set(0, 0, 2, *tl, 1.12)
            s.bonds_add(bonds)
            s.tab_bond_set(2, *tf)
            s.integrator_set(0.005)
            s.langevin_set(1, 1.0, 1.0, lexcl)
            s.capforce_set(_abi.CAP_COMPONENT, cap)
        else:
            s.vl(1.12, excl)
            r, e, f = tl
            _abi.call(s.lib, "espp_tab_pair_set", s.h, 0, 0, 2, len(r), _abi.dptr(r),
                      _abi.dptr(e), _abi.dptr(f), 1.12, 0.0)
            s.bonds(bonds)
            r, e, f = tf
            _abi.call(s.lib, "espp_tab_bond_set", s.h, 2, len(r), _abi.dptr(r), _abi.dptr(e),
                      _abi.dptr(f), math.inf, 0.0)
            s.integrator(0.005)
            s.langevin(1.0, 1.0, excl=lexcl)
            s.capforce(_abi.CAP_COMPONENT, cap)

    ref = Sim(oracle_lib(), box, 0.3, cg, seed=9)
    ref.add(ids, pos)
    ref.decompose()
    setup(ref, False)
    dd = SpatialDecomposition(box, 0.3, cg, 3, lib=oracle_lib(), seed=9)
    dd.add_particles(ids, pos)
    dd.decompose()
    setup(dd, True)
    for s in (ref, dd):
        s.run(80)
    assert dd.resorts == ref.num_resorts() > 0
    assert np.array_equal(dd.vl_pairs(), ref.pairs())
    for which in (_abi.IA_TAB_PAIR, _abi.IA_TAB_BOND):
        assert math.isclose(dd.energy(which), ref.energy(which), rel_tol=1e-9)
        assert math.isclose(dd.virial(which), ref.virial(which), rel_tol=1e-8)
    x, v, _, img = dd.get_particles(ids)
    xr, vr, _, ir = ref.particles(ids)
    assert np.max(np.abs(x - xr)) < 1e-8 and np.array_equal(img, ir)


def test_phase_entry_points_refuse_misuse():
    """espp_dd_step without a run in progress, a step past the run's end, a halo write
    to a particle that is not a halo copy: errors with the reason (oracle)."""
    ids, pos, vel, box = _fluid_inputs(6)
    cg = cell_grid(box, 1.5, SKIN)
    s = Sim(oracle_lib(), box, SKIN, cg)
    s.add(ids, pos, vel)
    s.decompose()
    s.vl(1.5)
    s.integrator(0.005)
    out = np.zeros(1)
    with pytest.raises(RuntimeError, match="no step of a decomposed run is pending"):
        _abi.call(s.lib, "espp_dd_step", s.h, 0, _abi.dptr(out))
    with pytest.raises(RuntimeError, match="no decomposed run in progress"):
        _abi.call(s.lib, "espp_dd_run_end", s.h)
    _abi.call(s.lib, "espp_dd_run_begin", s.h, 1, _abi.dptr(out))
    assert out[0] > 0.0
    _abi.call(s.lib, "espp_dd_step", s.h, 0, _abi.dptr(out))
    assert out[0] == 0.0  # the last step has no integrate1
    with pytest.raises(RuntimeError, match="no step of a decomposed run is pending"):
        _abi.call(s.lib, "espp_dd_step", s.h, 0, _abi.dptr(out))
    _abi.call(s.lib, "espp_dd_run_end", s.h)
    p = np.zeros(3)
    with pytest.raises(RuntimeError, match="not a halo particle"):
        _abi.call(s.lib, "espp_dd_write_halo", s.h, 1, _abi.i64ptr(ids[:1]), _abi.dptr(p))
    kind = ctypes.c_int32()
    _abi.call(s.lib, "espp_memory_space", ctypes.byref(kind))
    assert kind.value == 0


def _rank_fails(rank, world, port, out_dir, exchange):
    import torch.distributed as dist
    for p in (REPO, os.path.join(REPO, "tests")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from espressopp_b200.domain import TorchComm
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ids, pos, vel, box = _fluid_inputs(13)
        dd = _decomposed(ids, pos, vel, box, cell_grid(box, RC, SKIN), 4, comm=TorchComm(dist),
                         exchange=exchange)
        if rank == 1:  # this rank's step 7 raises, as a failing library call would
            real, count = dd._phase, [0]

            def failing(name, d, arg):
                if name == "espp_dd_step":
                    count[0] += 1
                    if count[0] == 7:
                        raise RuntimeError("injected failure")
                return real(name, d, arg)
            dd._phase = failing
        try:
            dd.run(20)
            msg = "no error"
        except RuntimeError as e:
            msg = str(e)
        with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
            f.write(msg)
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("exchange", ["host", "direct"])
def test_a_failing_rank_raises_on_every_rank(tmp_path, exchange):
    """Failure detection (esutil::Error, Error.cpp:52-64), made on the host: a library
    error on one rank in the middle of a run reaches both gloo ranks as the same error at
    the next gather, instead of leaving the other rank waiting."""
    port = _free_port()
    mp.start_processes(_rank_fails, args=(2, port, str(tmp_path), exchange), nprocs=2,
                       join=True, start_method="spawn")
    for r in range(2):
        msg = (tmp_path / ("rank%d.txt" % r)).read_text()
        assert "rank 1: injected failure" in msg


@pytest.mark.parametrize("h,slabs", [(1, 5), (2, "one cell each")])
def test_thin_and_uneven_slabs(h, slabs):
    """Slabs of one cell layer at halfCellInt 2 (each halo layer then comes from two
    neighbouring domains on either side) and uneven slabs (8 layers over 5 domains): the
    run equals one system's (oracle, direct halo refresh)."""
    rc = 1.5
    shift = 4.0 * (rc ** -12 - rc ** -6)
    pos, box = lattice(14, 0.8442, 0.05, 3)
    vel = mb_velocities(len(pos), 1.0, 4)
    ids = np.arange(len(pos), dtype=np.int64)
    cg = cell_grid(box, rc, SKIN, h)
    D = int(cg[2]) if slabs == "one cell each" else slabs
    ref = Sim(oracle_lib(), box, SKIN, cg, seed=4, half_cell_int=h)
    ref.add(ids, pos, vel)
    ref.decompose()
    ref.vl(rc)
    ref.lj(0, 0, 1.0, 1.0, rc, shift)
    ref.integrator(0.005)
    ref.langevin(1.0, 1.0)
    dd = SpatialDecomposition(box, SKIN, cg, D, lib=oracle_lib(), seed=4, half_cell_int=h,
                              exchange="direct")
    dd.add_particles(ids, pos, vel)
    dd.decompose()
    dd.vl_create(rc)
    dd.lj_set(0, 0, 1.0, 1.0, rc, shift)
    dd.integrator_set(0.005)
    dd.langevin_set(1, 1.0, 1.0)
    for s in (ref, dd):
        s.run(150)
    assert dd.resorts == ref.num_resorts() > 10
    assert dd.vl_digest() == ref.digest()
    assert np.max(np.abs(dd.get_particles(ids)[0] - ref.particles(ids)[0])) < 1e-9
