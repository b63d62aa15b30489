"""ParallelTempering on one GPU (src/ParallelTempering.py:78-203, src/MultiSystem.py).

The reference runs each replica on its own group of MPI ranks and swaps thermostat
temperatures between neighbours with a Metropolis test.  Here every replica is an
ordinary System on the same GPU; run() steps all of them with one graph launch
(espp_batch_run: one step loop per replica, no dependencies between them), and
exchange() applies the reference's rule unchanged.
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


class _MultiSystem:
    """The analysis hooks of MultiSystem that scripts call through pt._multisystem."""

    def __init__(self, pt):
        self._pt = pt

    def runAnalysisTemperature(self):
        return [a.compute() for a in self._pt._analysisT]

    def runAnalysisPotential(self):
        return [a.computeEnergy() for a in self._pt._analysisE]

    def runAnalysisNPart(self):
        return [int(a.compute()) for a in self._pt._analysisNPart]

    def runIntegrator(self, niter):
        self._pt.run(niter)


class ParallelTempering:
    """ParallelTempering(NumberOfSystems=4, RNG=None)."""

    def __init__(self, NumberOfSystems=4, RNG=None):
        if RNG is None:
            raise ValueError("ParallelTempering needs a random number generator")
        if NumberOfSystems < 2:
            raise ValueError("Parallel Tempering needs at least 2 systems to be able to work")
        self._RNG = RNG
        self._nsystems = int(NumberOfSystems)
        self._integrators = []
        self._thermostat = []
        self._analysisE = []
        self._analysisT = []
        self._analysisNPart = []
        self._oddeven = 0
        self._batch = None
        self._batch_members = None
        self._multisystem = _MultiSystem(self)

    def startDefiningSystem(self, n):
        if not 0 <= n < self._nsystems:
            raise ValueError("System number must be between 0 and %d" % self._nsystems)

    def endDefiningSystem(self, n):
        self.startDefiningSystem(n)

    def getNumberOfSystems(self):
        return self._nsystems

    def getNumberOfCPUsPerSystem(self):
        return 1

    def setIntegrator(self, integrator, thermostat):
        self._integrators.append(integrator)
        self._thermostat.append(thermostat)

    def setAnalysisE(self, analysisE):
        self._analysisE.append(analysisE)

    def setAnalysisT(self, analysisT):
        self._analysisT.append(analysisT)

    def setAnalysisNPart(self, analysisNPart):
        self._analysisNPart.append(analysisNPart)

    def _handles(self):
        return [integ.system.storage._h for integ in self._integrators]

    def run(self, nsteps):
        """Steps every replica nsteps with one graph launch."""
        if len(self._integrators) != self._nsystems:
            raise RuntimeError("%d of %d systems have an integrator" %
                               (len(self._integrators), self._nsystems))
        for integ in self._integrators:
            integ._push()
        lib = load_library()
        handles = self._handles()
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
        energies = self._multisystem.runAnalysisPotential()
        temperatures = self._multisystem.runAnalysisTemperature()
        nparts = self._multisystem.runAnalysisNPart()
        decisions = exchange_decisions(energies, temperatures, nparts, self._oddeven,
                                       self._RNG.random)
        for m, n, delta, metro, ok in decisions:
            log.info("systems %i and %i: dE=%10.5f random=%10.5f ==> exchange: %s", m, n, delta,
                     metro, "yes" if ok else "no")
            if ok:
                t1, t2 = temperatures[m], temperatures[n]
                self._thermostat[n].temperature = t1
                self._thermostat[m].temperature = t2
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
