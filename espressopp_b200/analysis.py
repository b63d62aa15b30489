"""Observables (src/analysis/Temperature.hpp:57-125, Pressure.cpp:41-119,
PressureTensor.hpp:51-80, RadialDistrF.cpp:47-150, NPart).  Reductions run on the GPU in
FP64."""
import ctypes

import numpy as np

from ._abi import call
from .core import Tensor


class _Observable:
    def __init__(self, system):
        self.system = system

    def _st(self):
        st = self.system.storage
        if st is None:
            raise RuntimeError("system has no storage")
        return st

    def _kinetic(self):
        st = self._st()
        v = ctypes.c_double()
        n = ctypes.c_int64()
        call(st._lib, "espp_kinetic", st._h, ctypes.byref(v), ctypes.byref(n))
        return v.value, n.value


class NPart(_Observable):
    def compute(self):
        return self._kinetic()[1]


class Temperature(_Observable):
    """T = sum m v^2 / (3 N), k_B = 1."""

    def compute(self):
        v2, n = self._kinetic()
        return v2 / (3.0 * n) if n else 0.0

    def compute_real(self):
        return self.compute()


class Pressure(_Observable):
    """P = (sum m v^2 + sum_interactions r.F) / (3 V)."""

    def compute(self):
        v2, _ = self._kinetic()
        w = sum(ia.computeVirial() for ia in self.system.shortRangeInteractions)
        L = self.system.bc.boxL
        return (v2 + w) / (3.0 * L[0] * L[1] * L[2])


class PressureTensor(_Observable):
    """P_ab = (sum m v_a v_b + W_ab) / V; kinetic part from the particle velocities."""

    def compute(self):
        st = self._st()
        _, pos, vel, _, _ = st.getAll()
        masses = np.array([st._masses[i] for i in sorted(st._types)])
        vv = np.zeros(6)
        mv = vel * masses[:, None]
        vv[0] = np.sum(mv[:, 0] * vel[:, 0])
        vv[1] = np.sum(mv[:, 1] * vel[:, 1])
        vv[2] = np.sum(mv[:, 2] * vel[:, 2])
        vv[3] = np.sum(mv[:, 0] * vel[:, 1])
        vv[4] = np.sum(mv[:, 0] * vel[:, 2])
        vv[5] = np.sum(mv[:, 1] * vel[:, 2])
        w = np.zeros(6)
        for ia in self.system.shortRangeInteractions:
            w += np.asarray(ia.computeVirialTensor())
        L = self.system.bc.boxL
        return Tensor((vv + w) / (L[0] * L[1] * L[2]))


class RadialDistrF(_Observable):
    """analysis.RadialDistrF(system) (RadialDistrF.py:45-60, RadialDistrF.cpp:47-150):
    compute(rdfN) returns the radial distribution function of the current configuration
    in rdfN bins up to half the y edge of the box, computed on the GPU over all pairs."""

    print_progress = False

    def compute(self, rdfN):
        st = self._st()
        out = np.zeros(int(rdfN))
        call(st._lib, "espp_rdf", st._h, int(rdfN), out.ctypes.data_as(
            ctypes.POINTER(ctypes.c_double)))
        return list(out)
