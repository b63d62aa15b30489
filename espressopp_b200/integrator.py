"""Integrator and extensions of the drop-in API.

VelocityVerlet (src/integrator/VelocityVerlet.cpp:63-437, VelocityVerlet.py:39-49),
LangevinThermostat (LangevinThermostat.cpp:41-233, LangevinThermostat.py:59-75) and
CapForce (CapForce.cpp:34-255).  The whole step runs on the GPU; run(n) pushes the
current parameters and extensions to the system handle and steps it n times.
"""
import ctypes

import numpy as np

from . import _abi
from ._abi import call, dptr, i64ptr


class Extension:
    """integrator.Extension (src/integrator/Extension.cpp:30-44)."""

    def __init__(self, system):
        self.system = system
        self.integrator = None

    def setIntegrator(self, integrator):
        self.integrator = integrator

    def connect(self):
        self._connected = True

    def disconnect(self):
        self._connected = False


class LangevinThermostat(Extension):
    """integrator.LangevinThermostat(system): F += -gamma m v + sqrt(24 T gamma / dt)
    (U - 0.5) sqrt(m) after the force calculation.  The uniform U comes from a
    Philox4x32-10 stream keyed on (rng seed, particle id) and counted by step."""

    def __init__(self, system):
        Extension.__init__(self, system)
        if system.rng is None:
            raise RuntimeError("system has no RNG")
        self.gamma = 0.0
        self.temperature = 0.0
        self.adress = False
        self._excl = []
        self._connected = True

    def addExclpid(self, pid):
        self._excl.append(int(pid))

    def addExclusions(self, pids):
        for p in pids:
            self.addExclpid(p)

    def _push(self, st):
        ex = np.ascontiguousarray(self._excl, np.int64)
        on = 1 if (self._connected and (self.gamma != 0.0 or self.temperature != 0.0)) else 0
        call(st._lib, "espp_langevin_set", st._h, on, float(self.gamma),
             float(self.temperature), len(ex), i64ptr(ex) if len(ex) else None)


class CapForce(Extension):
    """integrator.CapForce(system, capForce, particleGroup=None) (CapForce.cpp:38-102,
    170-200): a scalar caps |F| (absolute capping), a 3-vector caps each component; the
    kind is fixed by the constructor, the setters change the values."""

    def __init__(self, system, capForce, particleGroup=None):
        Extension.__init__(self, system)
        if particleGroup is not None:
            raise NotImplementedError("CapForce on a particle group is not supported")
        self._absCapping = bool(np.isscalar(capForce))
        self._absCapForce = float(capForce) if self._absCapping else 0.0
        self._capForce = (np.zeros(3) if self._absCapping
                          else np.asarray(tuple(capForce), np.float64))
        self._connected = True

    @property
    def capForce(self):
        return self._absCapForce if self._absCapping else tuple(self._capForce)

    def setCapForce(self, capForce):
        self._capForce = np.asarray(tuple(capForce), np.float64)

    def setAbsCapForce(self, absCapForce):
        self._absCapForce = float(absCapForce)

    def getCapForce(self):
        from .core import Real3D
        return Real3D(self._capForce)

    def getAbsCapForce(self):
        return self._absCapForce

    def _push(self, st):
        if not self._connected:
            call(st._lib, "espp_capforce_set", st._h, _abi.CAP_OFF, None)
            return
        if self._absCapping:
            cap = np.array([self._absCapForce] * 3)
            mode = _abi.CAP_ABS
        else:
            cap = np.ascontiguousarray(self._capForce, np.float64)
            mode = _abi.CAP_COMPONENT
        call(st._lib, "espp_capforce_set", st._h, mode, dptr(cap))


class MDIntegrator:
    """integrator.MDIntegrator (src/integrator/MDIntegrator.cpp:40-107)."""

    def __init__(self, system):
        self.system = system
        self._dt = 0.005
        self._step = 0
        self._ext = []

    @property
    def dt(self):
        return self._dt

    @dt.setter
    def dt(self, v):
        if float(v) == 0.0:
            raise ValueError("Timestep 'dt' must be non-zero!")
        self._dt = float(v)

    @property
    def step(self):
        st = self.system.storage
        if st is not None and st._h:
            v = ctypes.c_int64()
            call(st._lib, "espp_step_get", st._h, ctypes.byref(v))
            self._step = v.value
        return self._step

    @step.setter
    def step(self, v):
        self._step = int(v)
        st = self.system.storage
        if st is not None and st._h:
            call(st._lib, "espp_step_set", st._h, self._step)

    def addExtension(self, extension):
        extension.setIntegrator(self)
        extension.connect()
        self._ext.append(extension)
        return len(self._ext) - 1

    def getExtension(self, k):
        return self._ext[k]

    def getNumberOfExtensions(self):
        return len(self._ext)


class VelocityVerlet(MDIntegrator):
    """integrator.VelocityVerlet(system)."""

    def __init__(self, system):
        MDIntegrator.__init__(self, system)
        self._timers = (0.0,) * 10

    def _push(self):
        st = self.system.storage
        if st is None:
            raise RuntimeError("system has no storage")
        call(st._lib, "espp_integrator_set", st._h, self._dt)
        lang = [e for e in self._ext if isinstance(e, LangevinThermostat)]
        caps = [e for e in self._ext if isinstance(e, CapForce)]
        if len(lang) > 1 or len(caps) > 1:
            raise NotImplementedError("at most one Langevin thermostat and one CapForce")
        if lang:
            lang[0]._push(st)
        else:
            call(st._lib, "espp_langevin_set", st._h, 0, 0.0, 0.0, 0, None)
        if caps:
            caps[0]._push(st)
        else:
            call(st._lib, "espp_capforce_set", st._h, _abi.CAP_OFF, None)
        return st

    def run(self, nsteps):
        st = self._push()
        call(st._lib, "espp_run", st._h, int(nsteps))
        t = np.zeros(10)
        call(st._lib, "espp_timers", st._h, dptr(t))
        self._timers = tuple(float(x) for x in t)

    def getNumResorts(self):
        st = self.system.storage
        v = ctypes.c_int64()
        call(st._lib, "espp_num_resorts", st._h, ctypes.byref(v))
        return v.value

    def getTimers(self):
        """(run, pair, FENE, angle, comm1, comm2, int1, int2, resort, other) seconds."""
        return [self._timers]

    def resetTimers(self):
        self._timers = (0.0,) * 10

    def printTimers(self):
        names = ["run", "pair", "FENE", "angle", "comm1", "comm2", "int1", "int2", "resort",
                 "other"]
        for n, v in zip(names, self._timers):
            print("%s = %.3f" % (n, v))
