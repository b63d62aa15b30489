"""ParallelTempering (src/ParallelTempering.py:78-203, src/MultiSystem.py).

The reference runs each replica on its own group of MPI ranks and swaps thermostat
temperatures between neighbours with a Metropolis test.  Here every replica is an
ordinary System on a GPU; run() steps a rank's replicas with one graph launch
(espp_batch_run: one step loop per replica, no dependencies between them), and
exchange() applies the reference's rule unchanged.

With a torch.distributed process group (one process per GPU) the replicas are shared
out among the ranks by particle count (partition_replicas), each rank steps only its
own, and exchange() gathers (E_pot, T, N) of every replica with one all-reduce of an
R x 3 FP64 array; every rank then takes the same Metropolis decisions from the same
random stream (the reference draws them on every rank of its MultiSystem from the
same seed) and sets the temperatures of its own replicas.
"""
import ctypes
import logging
from math import exp

from ._abi import call
from ._lib import load_library

log = logging.getLogger(__name__)


def exchange_decisions(energies, temperatures, nparts, oddeven, uniform):
    """The Metropolis rule of ParallelTempering.exchange (ParallelTempering.py:164-203).

    Neighbours (m, m+1) with m = 2 i + oddeven are tested with
    delta = (1/t2 - 1/t1) (e1/n1 - e2/n2); they swap when delta <= 0 or
    exp(-delta) > u, u drawn from ``uniform()`` for every tested pair.  Returns
    (m, n, delta, u, accepted) for each tested pair."""
    out = []
    for i in range(len(energies) // 2):
        m = 2 * i + oddeven
        n = m + 1
        if n < len(energies):
            metro = uniform()
            t1, t2 = temperatures[m], temperatures[n]
            e1, e2 = energies[m], energies[n]
            n1, n2 = nparts[m], nparts[n]
            delta = (1 / t2 - 1 / t1) * (e1 / n1 - e2 / n2)
            accepted = delta <= 0 or exp(-delta) > metro
            out.append((m, n, delta, metro, accepted))
    return out


def partition_replicas(sizes, world):
    """Owner rank of each replica: longest-processing-time assignment by particle count
    (largest first, each to the rank with the fewest particles so far, ties to the lower
    rank).  Deterministic: every rank computes the same table."""
    order = sorted(range(len(sizes)), key=lambda r: (-int(sizes[r]), r))
    load = [0] * world
    owner = [0] * len(sizes)
    for r in order:
        k = min(range(world), key=lambda q: (load[q], q))
        owner[r] = k
        load[k] += int(sizes[r])
    return owner


def gather_replica_rows(rows, nreplicas, group=None):
    """(E_pot, T, N) of every replica from each rank's own rows {replica: (E, T, N)}:
    one all-reduce (sum) of an R x 3 FP64 array in which each rank fills its rows.
    Without a group the rows are all local."""
    import numpy as np
    out = np.zeros((nreplicas, 3))
    for n, r in rows.items():
        out[n] = r
    if group is None:
        return out
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(out).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


class _MultiSystem:
    """The analysis hooks of MultiSystem that scripts call through pt._multisystem: values
    of every replica, in replica order (gathered from the ranks that own them)."""

    def __init__(self, pt):
        self._pt = pt

    def _rows(self):
        pt = self._pt
        rows = {}
        for n in pt._local:
            rows[n] = (pt._analysisE[n].computeEnergy() if n in pt._analysisE else 0.0,
                       pt._analysisT[n].compute() if n in pt._analysisT else 0.0,
                       float(pt._analysisNPart[n].compute()) if n in pt._analysisNPart else 0.0)
        return gather_replica_rows(rows, pt._nsystems, pt._group)

    def runAnalysisTemperature(self):
        return [float(v) for v in self._rows()[:, 1]]

    def runAnalysisPotential(self):
        return [float(v) for v in self._rows()[:, 0]]

    def runAnalysisNPart(self):
        return [int(v) for v in self._rows()[:, 2]]

    def runIntegrator(self, niter):
        self._pt.run(niter)


class ParallelTempering:
    """ParallelTempering(NumberOfSystems=4, RNG=None[, group, sizes]).

    group: a torch.distributed process group over which the replicas are shared out (one
    process per GPU); None keeps them all in this process.  sizes: particle counts of the
    replicas, used to balance the ranks (otherwise replica n goes to rank n % world).
    startDefiningSystem(n) returns whether this rank owns replica n; a script may skip
    building the replicas it does not own, and the set-up calls for them are ignored."""

    def __init__(self, NumberOfSystems=4, RNG=None, group=None, sizes=None):
        if RNG is None:
            raise ValueError("ParallelTempering needs a random number generator")
        if NumberOfSystems < 2:
            raise ValueError("Parallel Tempering needs at least 2 systems to be able to work")
        self._RNG = RNG
        self._nsystems = int(NumberOfSystems)
        self._group = group
        if group is not None:
            import torch.distributed as dist
            self._rank = dist.get_rank(group)
            world = dist.get_world_size(group)
        else:
            self._rank, world = 0, 1
        if sizes is not None:
            if len(sizes) != self._nsystems:
                raise ValueError("sizes needs one particle count per system")
            self._owner = partition_replicas(sizes, world)
        else:
            self._owner = [n % world for n in range(self._nsystems)]
        self._local = [n for n in range(self._nsystems) if self._owner[n] == self._rank]
        self._current = None
        self._integ = {}
        self._thermo = {}
        self._analysisE = {}
        self._analysisT = {}
        self._analysisNPart = {}
        self._oddeven = 0
        self._batch = None
        self._batch_members = None
        self._multisystem = _MultiSystem(self)

    def isLocal(self, n):
        return self._owner[n] == self._rank

    def startDefiningSystem(self, n):
        if not 0 <= n < self._nsystems:
            raise ValueError("System number must be between 0 and %d" % self._nsystems)
        self._current = n
        return self.isLocal(n)

    def endDefiningSystem(self, n):
        if not 0 <= n < self._nsystems:
            raise ValueError("System number must be between 0 and %d" % self._nsystems)
        self._current = None

    def getNumberOfSystems(self):
        return self._nsystems

    def getNumberOfCPUsPerSystem(self):
        return 1

    def _slot(self, table):
        n = self._current if self._current is not None else len(table)
        return n if self.isLocal(n) else None

    def setIntegrator(self, integrator, thermostat):
        n = self._slot(self._integ)
        if n is not None:
            self._integ[n] = integrator
            self._thermo[n] = thermostat

    def setAnalysisE(self, analysisE):
        n = self._slot(self._analysisE)
        if n is not None:
            self._analysisE[n] = analysisE

    def setAnalysisT(self, analysisT):
        n = self._slot(self._analysisT)
        if n is not None:
            self._analysisT[n] = analysisT

    def setAnalysisNPart(self, analysisNPart):
        n = self._slot(self._analysisNPart)
        if n is not None:
            self._analysisNPart[n] = analysisNPart

    @property
    def _integrators(self):
        return [self._integ[n] for n in sorted(self._integ)]

    @property
    def _thermostat(self):
        """This rank's thermostats, in replica order (all of them without a group)."""
        return [self._thermo[n] for n in sorted(self._thermo)]

    def _handles(self):
        return [self._integ[n].system.storage._h for n in sorted(self._integ)]

    def run(self, nsteps):
        """Steps this rank's replicas nsteps with one graph launch."""
        if sorted(self._integ) != self._local:
            raise RuntimeError("%d of the %d systems of this rank have an integrator" %
                               (len(self._integ), len(self._local)))
        for n in sorted(self._integ):
            self._integ[n]._push()
        lib = load_library()
        handles = self._handles()
        if not handles:
            return
        key = tuple(h.value for h in handles)
        if self._batch is None or self._batch_members != key:
            self._free_batch()
            arr = (ctypes.c_void_p * len(handles))(*[h.value for h in handles])
            self._batch = ctypes.c_void_p()
            call(lib, "espp_batch_create", arr, len(handles), ctypes.byref(self._batch))
            self._batch_members = key
        call(lib, "espp_batch_run", self._batch, int(nsteps))

    def last_run_ms(self):
        v = ctypes.c_double()
        call(load_library(), "espp_batch_last_run_ms", self._batch, ctypes.byref(v))
        return v.value

    def exchange(self):
        """One replica-exchange attempt between neighbours (odd/even alternating)."""
        self._oddeven = 1 if self._oddeven == 0 else 0
        rows = self._multisystem._rows()
        energies = [float(v) for v in rows[:, 0]]
        temperatures = [float(v) for v in rows[:, 1]]
        nparts = [int(v) for v in rows[:, 2]]
        decisions = exchange_decisions(energies, temperatures, nparts, self._oddeven,
                                       self._RNG.random)
        for m, n, delta, metro, ok in decisions:
            log.info("systems %i and %i: dE=%10.5f random=%10.5f ==> exchange: %s", m, n, delta,
                     metro, "yes" if ok else "no")
            if ok:
                t1, t2 = temperatures[m], temperatures[n]
                if n in self._thermo:
                    self._thermo[n].temperature = t1
                if m in self._thermo:
                    self._thermo[m].temperature = t2
        return decisions

    def _free_batch(self):
        if self._batch is not None and self._batch.value:
            load_library().espp_batch_destroy(self._batch)
        self._batch = None

    def __del__(self):
        try:
            self._free_batch()
        except Exception:
            pass
