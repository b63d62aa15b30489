"""Observables (src/analysis/Temperature.hpp:57-125, Pressure.cpp:41-119,
PressureTensor.hpp:51-80, RadialDistrF.cpp:47-150, NPart, ConfigsParticleDecomp.cpp,
MeanSquareDispl.cpp).  Reductions run on the GPU in FP64."""
import ctypes

import numpy as np

from ._abi import call
from .core import Real3D, Tensor


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
    """T = sum m v^2 / (3 N), k_B = 1 (Temperature.hpp:57-126), reduced on the GPU in
    FP64.  After add_type, only particles of the added types count (valid_type_ids):
    types 0..63 are selected by a bit mask inside the same device reduction; a larger
    type id is summed from one state download.  With no (selected) particle the result
    is sumT / (3 * 0) = nan, as in the reference.  getEkin returns 0.5 sum m v^2 of the
    last compute."""

    def __init__(self, system):
        _Observable.__init__(self, system)
        self._valid_types = set()
        self._ekin = 0.0

    def add_type(self, type_id):
        self._valid_types.add(int(type_id))

    def remove_type(self, type_id):
        if int(type_id) in self._valid_types:
            self._valid_types.discard(int(type_id))
            return True
        return False

    def _typed(self):
        st = self._st()
        if all(0 <= t < 64 for t in self._valid_types):
            mask = 0
            for t in self._valid_types:
                mask |= 1 << t
            v = ctypes.c_double()
            n = ctypes.c_int64()
            call(st._lib, "espp_kinetic_types", st._h, ctypes.c_uint64(mask), ctypes.byref(v),
                 ctypes.byref(n))
            return v.value, n.value
        ids, _, vel, _, _ = st.getAll()
        types = np.array([st._types[int(p)] for p in ids], np.int64)
        masses = np.array([st._masses[int(p)] for p in ids], np.float64)
        sel = np.isin(types, np.array(sorted(self._valid_types), np.int64))
        return float(np.sum(masses[sel] * np.sum(vel[sel] ** 2, axis=1))), int(sel.sum())

    def compute(self):
        v2, n = self._typed() if self._valid_types else self._kinetic()
        self._ekin = 0.5 * v2
        return v2 / (3.0 * n) if n else float("nan")

    def compute_real(self):
        return self.compute()

    def getEkin(self):
        return self._ekin


class Pressure(_Observable):
    """P = (sum m v^2 + sum_interactions r.F) / (3 V)."""

    def compute(self):
        v2, _ = self._kinetic()
        w = sum(ia.computeVirial() for ia in self.system.shortRangeInteractions)
        L = self.system.bc.boxL
        return (v2 + w) / (3.0 * L[0] * L[1] * L[2])


class PressureTensor(_Observable):
    """P_ab = (sum m v_a v_b + W_ab) / V (PressureTensor.hpp:51-80); the kinetic sum and
    the virials are reduced on the GPU.  performMeasurement / getAverageValue / reset /
    getNumberOfMeasurements keep the reference's running average and variance
    (PressureTensor.hpp:96-143, Knuth's update): getAverageValue returns the six averages
    followed by the six standard deviations sqrt(M2 / (n - 1))."""

    def __init__(self, system):
        _Observable.__init__(self, system)
        self.reset()

    def reset(self):
        self._n = 0
        self._avg = np.zeros(6)
        self._m2 = np.zeros(6)

    def performMeasurement(self):
        res = np.asarray(self.compute(), np.float64)
        self._n += 1
        if self._n == 1:
            self._avg = res.copy()
        else:
            new = self._avg + (res - self._avg) / self._n
            self._m2 = self._m2 + (res - self._avg) * (res - new)
            self._avg = new

    def getNumberOfMeasurements(self):
        return self._n

    def getAverageValue(self):
        if self._n == 0:
            return [0.0] * 12
        std = [float(np.sqrt(v / (self._n - 1))) if self._n > 1 else float("nan")
               for v in self._m2]
        return [float(a) for a in self._avg] + std

    def compute(self):
        st = self._st()
        vv = np.zeros(6)
        call(st._lib, "espp_kinetic_tensor", st._h,
             vv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
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


class Configuration:
    """One snapshot (analysis/Configuration.cpp:103-240): values by particle id."""

    def __init__(self, ids, xyz, vel=None, force=None, radius=None):
        self._ids = [int(i) for i in ids]
        self._index = {pid: k for k, pid in enumerate(self._ids)}
        self._xyz = None if xyz is None else np.asarray(xyz, np.float64).reshape(-1, 3)
        self._vel = None if vel is None else np.asarray(vel, np.float64).reshape(-1, 3)
        self._frc = None if force is None else np.asarray(force, np.float64).reshape(-1, 3)
        self._rad = None if radius is None else np.asarray(radius, np.float64).reshape(-1)

    def _row(self, a, pid, what):
        if a is None:
            raise RuntimeError("configuration has no %s" % what)
        return Real3D(a[self._index[int(pid)]])

    def getCoordinates(self, pid):
        return self._row(self._xyz, pid, "coordinates")

    __getitem__ = getCoordinates

    def getVelocities(self, pid):
        return self._row(self._vel, pid, "velocities")

    def getForces(self, pid):
        return self._row(self._frc, pid, "forces")

    def getRadius(self, pid):
        if self._rad is None:
            raise RuntimeError("configuration has no radius")
        return float(self._rad[self._index[int(pid)]])

    def getIds(self):
        return list(self._ids)

    def __iter__(self):
        return iter(self._ids)

    @property
    def size(self):
        return len(self._ids)


class Configurations(_Observable):
    """analysis.Configurations(system, pos=True, vel=False, force=False, radius=False,
    folded=True) (src/analysis/Configurations.{py,cpp}): a trajectory of snapshots of all
    particles, kept on the host.  Positions are folded into the box (BC::foldPosition) or
    unfolded with their images (BC::unfoldPosition).  `capacity` 0 keeps every snapshot;
    otherwise the oldest is dropped before a new one is added.  `[n]` counts back from the
    newest snapshot (Configurations::get); iteration runs from the oldest.  The radius is
    the reference's default particle radius, 1.0, since the GPU storage holds none."""

    def __init__(self, system, pos=True, vel=False, force=False, radius=False, folded=True):
        _Observable.__init__(self, system)
        self._pos, self._vel, self._force, self._radius = pos, vel, force, radius
        self.folded = folded
        self._confs = []
        self._cap = 0

    @property
    def capacity(self):
        return self._cap

    @capacity.setter
    def capacity(self, max_configs):
        max_configs = int(max_configs)
        if max_configs < 0:
            return  # the reference logs an error and keeps its capacity
        self._cap = max_configs
        if max_configs and len(self._confs) > max_configs:
            del self._confs[:len(self._confs) - max_configs]

    @property
    def size(self):
        return len(self._confs)

    def gather(self):
        ids, pos, vel, frc, img = self._st().getAll()
        xyz = None
        if self._pos:
            L = np.asarray(self.system.bc.boxL, np.float64)
            if self.folded:
                t = np.floor(pos * (1.0 / L))
                xyz = pos - t * L
            else:
                xyz = pos + img * L
        conf = Configuration(ids, xyz, vel if self._vel else None,
                             frc if self._force else None,
                             np.ones(len(ids)) if self._radius else None)
        if self._cap and len(self._confs) >= self._cap:
            del self._confs[0]
        self._confs.append(conf)

    def __getitem__(self, stackpos):
        n = len(self._confs)
        if 0 <= stackpos < n:
            return self._confs[n - 1 - stackpos]
        return None  # Configurations::get <out-of-range>: a null configuration

    def back(self):
        return self._confs[-1]

    def all(self):
        return list(self._confs)

    def __iter__(self):
        return iter(list(self._confs))

    def clear(self):
        self._confs = []


class ConfigsParticleDecomp(_Observable):
    """analysis.ConfigsParticleDecomp(system[, chainlength, start_pid])
    (ConfigsParticleDecomp.py:40-90, ConfigsParticleDecomp.hpp:61-230): a list of
    snapshots of the particles present at construction (or, with chainlength, of the ids
    start_pid .. start_pid + N - 1), held on the GPU.  key selects what a snapshot holds:
    "position", "velocity" or "unfolded" (position + image * box)."""

    key = "position"
    _KEYS = {"position": 0, "velocity": 1, "unfolded": 2}

    def __init__(self, system, chainlength=None, start_pid=0):
        super().__init__(system)
        st = self._st()
        if self.key not in self._KEYS:
            raise RuntimeError("Error. Key %s is unknown. Use position, unfolded or velocity."
                               % self.key)
        n = st.getNRealParticles()
        if chainlength is None:
            ids = st.getRealParticleIDs()
        else:
            if n % int(chainlength) != 0:
                print("chainlength does not match total number of particles\n"
                      "chainlength: %d\n num_of_part %d\n" % (chainlength, n))
            ids = list(range(int(start_pid), int(start_pid) + n))
        self.chainlength = None if chainlength is None else int(chainlength)
        self.start_pid = int(start_pid)
        self.num_of_part = n
        self._ids = np.ascontiguousarray(ids, np.int64)
        self._lib = st._lib
        h = ctypes.c_void_p()
        call(self._lib, "espp_confs_create", st._h, self._KEYS[self.key], len(self._ids),
             self._ids.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.espp_confs_destroy(h)
            self._h = None

    def gather(self):
        call(self._lib, "espp_confs_gather", self._h)

    def gatherFromFile(self, filename):
        """Reads "id type x y z" lines after two header lines (ConfigsParticleDecomp.cpp:144-206)."""
        try:
            with open(filename) as f:
                lines = f.read().splitlines()[2:]
        except OSError:
            raise RuntimeError("Unable to open file %s" % filename)
        conf = {}
        for line in lines:
            parts = line.split()
            if len(parts) >= 5:
                conf[int(parts[0])] = (float(parts[2]), float(parts[3]), float(parts[4]))
        print("read %d particles from file %s" % (len(conf), filename))
        if len(conf) != self.num_of_part:
            raise RuntimeError("Number of read particles does not match the number of particles "
                               "of the system (which is %d)" % self.num_of_part)
        xyz = np.array([conf[int(pid)] for pid in self._ids], np.float64).reshape(-1)
        call(self._lib, "espp_confs_push", self._h,
             xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def clear(self):
        call(self._lib, "espp_confs_clear", self._h)

    @property
    def size(self):
        m = ctypes.c_int32()
        call(self._lib, "espp_confs_size", self._h, ctypes.byref(m))
        return m.value

    def __getitem__(self, m):
        out = np.zeros(3 * len(self._ids))
        call(self._lib, "espp_confs_get", self._h, int(m),
             out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return Configuration(self._ids, out)

    def all(self):
        return [self[m] for m in range(self.size)]

    def __iter__(self):
        return iter(self.all())

    def compute(self):
        raise NotImplementedError("compute() is defined by the derived analyses")


class MeanSquareDispl(ConfigsParticleDecomp):
    """analysis.MeanSquareDispl(system[, chainlength, start_pid]) (MeanSquareDispl.py:50-80,
    MeanSquareDispl.cpp): snapshots of unfolded positions; compute() returns, for every lag
    m, the mean over snapshot pairs and particles of |r(t) - r(t+m)|^2 / 6; computeG3() the
    same for the centres of mass of the chains relative to their snapshot's mean.  The lag
    sums run on the GPU in FP64."""

    key = "unfolded"

    def __init__(self, system, chainlength=None, start_pid=0):
        super().__init__(system, chainlength, start_pid)
        self.print_progress = True

    def _progress_done(self):
        print("calculation progress (mean square displacement): 100%")

    def compute(self):
        out = np.zeros(self.size)
        call(self._lib, "espp_msd", self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        self._progress_done()
        return list(out)

    def computeG2(self):
        print("Sorry. Computation of G2 does not work correctly.", end="")
        print("Update ESPResSO++ when it is repaired. ")
        return []

    def computeG3(self):
        if self.chainlength is None:
            raise RuntimeError("computeG3 needs the chainlength given at construction")
        out = np.zeros(self.size)
        call(self._lib, "espp_msd_chain_com", self._h, self.chainlength,
             out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        self._progress_done()
        return list(out)

    def strange(self):
        print(1)
        return 1
