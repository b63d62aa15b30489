"""Failure paths on the GPU, made to happen without faulting it: a Verlet list that
outgrows its capacity inside the captured step-loop graph, coordinates that leave the box
for good, and a bounded device wait that runs out."""
import ctypes
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import Sim, cell_grid, cuda_lib, lattice, oracle_lib

pytestmark = pytest.mark.gpu

RC, SKIN, SIG = 2.5, 0.3, 0.8


def _implosion():
    """A dilute LJ gas (rho 0.3) whose x and y velocities all point at the box axis:
    by step 100 the densest particles have ~4x the neighbours of the start."""
    pos, box = lattice(12, 0.3, 0.05, seed=3)
    vel = np.zeros_like(pos)
    vel[:, :2] = -(pos[:, :2] - box[0] / 2)
    return np.arange(len(pos)), pos, vel, box


def _setup(lib, prec, pid, pos, vel, box):
    s = Sim(lib, box, SKIN, cell_grid(box, RC, SKIN), precision=prec)
    s.add(pid, pos, vel)
    s.decompose()
    s.vl(RC)
    s.lj(0, 0, 1.0, SIG, RC, 4.0 * ((SIG / RC) ** 12 - (SIG / RC) ** 6))
    s.integrator(0.005)
    return s


def _initial_capacity(n, box):
    """The list capacity a system starts with: 1.6x the neighbours expected at the mean
    density, plus 32, in blocks of 8."""
    rho = n / np.prod(box)
    k = math.ceil(rho * 4.0 / 3.0 * math.pi * (RC + SKIN) ** 3 * 1.6) + 32
    return (k + 7) // 8 * 8


def _max_neighbours(pos, box):
    d = pos[:, None, :] - pos[None, :, :]
    d -= box * np.round(d / box)
    return int(((d ** 2).sum(-1) < (RC + SKIN) ** 2).sum(1).max()) - 1


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_list_overflow_inside_graph_recovers(prec, monkeypatch):
    """The graph's list build overflows mid-run; the run is rolled back to its start,
    the capacity grows and the steps are taken again on the host loop.  Builds fall on
    the same steps as in a host-loop run.  The list rebuilt at the restored positions
    holds the same pairs inside the cutoff in another order, so the trajectories agree to
    the rounding of the per-particle sums (FP32 in the mixed mode, grown by the collision's
    chaos over 110 steps), and the FP64 one follows the oracle.  The first run (40 steps)
    stays inside the initial capacity, so the second starts from a list built steps
    earlier."""
    pid, pos, vel, box = _implosion()
    tol = 1e-3 if prec == _abi.PREC_MIXED else 1e-9
    sims = []
    for graph in ("0", "1"):
        monkeypatch.setenv("ESPP_B200_GRAPH", graph)
        s = _setup(cuda_lib(), prec, pid, pos, vel, box)
        s.run(40)
        s.run(110)
        sims.append(s)
    a, b = sims[0].particles(pid), sims[1].particles(pid)
    assert _max_neighbours(a[0], box) > _initial_capacity(len(pid), box) + 40
    assert np.max(np.abs(a[0] - b[0])) <= tol
    assert np.max(np.abs(a[1] - b[1])) <= 100 * tol
    assert sims[0].builds() == sims[1].builds()
    assert sims[0].step() == sims[1].step() == 150
    # the graph is captured again at the larger capacity and keeps matching
    for s in sims:
        s.run(20)
    a, b = sims[0].particles(pid), sims[1].particles(pid)
    assert np.max(np.abs(a[0] - b[0])) <= tol
    assert sims[0].builds() == sims[1].builds()
    if prec == _abi.PREC_FP64:
        o = _setup(oracle_lib(), _abi.PREC_FP64, pid, pos, vel, box)
        for n in (40, 110, 20):
            o.run(n)
        ref = o.particles(pid)
        assert np.max(np.abs(b[0] - ref[0])) < 1e-8
        assert np.array_equal(b[3], ref[3])
        assert o.builds() == sims[1].builds()


@pytest.mark.parametrize("bad", [math.nan, math.inf, 1.0e12])
def test_particle_in_outer_space_raises(bad):
    """A coordinate that no fold brings back into the box is an error (Storage::decompose,
    'particle ... has moved to outer space').  For NaN the oracle agrees; for an infinite
    coordinate or one more than 1e9 box lengths away the reference's fold converts a value
    outside the int range (undefined behaviour, a silent wrong image on x86), so only the
    GPU's stricter answer is checked there."""
    pos, box = lattice(10, 0.8442, 0.05, seed=1)
    pos[17, 1] = bad
    pid = np.arange(len(pos))
    libs = (oracle_lib(), cuda_lib()) if math.isnan(bad) else (cuda_lib(),)
    for lib in libs:
        s = Sim(lib, box, SKIN, cell_grid(box, RC, SKIN), precision=_abi.PREC_FP64)
        s.add(pid, pos)
        with pytest.raises(RuntimeError, match="outer space"):
            s.decompose()


def test_bounded_wait_times_out_and_the_system_stays_usable():
    """An mbarrier wait that nothing completes gives up after its tries, sets the error
    status the host reads, releases its TMEM; the same system then steps normally."""
    pid = np.arange(1000)
    pos, box = lattice(10, 0.8442, 0.05, seed=1)
    sims = [_setup(lib, _abi.PREC_FP64, pid, pos, np.zeros_like(pos), box)
            for lib in (oracle_lib(), cuda_lib())]
    g = sims[1]
    ns = ctypes.c_double()
    for spins in (1, 4096):
        rc = g.lib.espp_selftest_bounded_wait(g.h, spins, ctypes.byref(ns))
        assert rc == -7, _abi.last_error(g.lib)
        assert "bounded wait" in _abi.last_error(g.lib)
    # 4096 tries: the wait takes measurable time and ends well inside a second
    assert 0.0 < ns.value < 1.0e9
    for s in sims:
        s.run(10)
    a, b = sims[0].particles(pid), sims[1].particles(pid)
    assert np.max(np.abs(a[0] - b[0])) < 1e-9
