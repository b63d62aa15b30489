"""Potentials and interaction templates of the drop-in API.

LennardJones / LennardJonesCapped / FENE hold parameters and evaluate themselves on the
host for single distances (as the reference's Python potentials do); the interaction
objects push their parameters to the GPU system when they are added to the system.
References: src/interaction/Potential.hpp:190-431, LennardJones.hpp:43-174,
LennardJonesCapped.hpp:80-160, FENE.hpp:35-115, VerletListInteractionTemplate.hpp,
FixedPairListInteractionTemplate.hpp, and the Python wrappers LennardJones.py:719-760,
FENE.py:98-141.
"""
import ctypes
import math

from . import _abi
from ._abi import call, dptr
from .core import Real3D, Tensor, infinity

ROUND_ERROR_PREC = 2.220446049250313e-16


class Potential:
    """PotentialTemplate cutoff/shift plumbing (Potential.hpp:190-431)."""

    def __init__(self, cutoff, shift):
        self._cutoff = float(cutoff)
        self._auto = shift == "auto"
        self._shift = 0.0 if self._auto else float(shift)
        self._update_shift()

    def _update_shift(self):
        if self._auto:
            cs = self._cutoff * self._cutoff
            self._shift = 0.0 if math.isinf(cs) else self._energy_raw(cs)

    @property
    def cutoff(self):
        return self._cutoff

    @cutoff.setter
    def cutoff(self, v):
        self._cutoff = float(v)
        self._update_shift()

    @property
    def shift(self):
        return self._shift

    @shift.setter
    def shift(self, v):
        if v == "auto":
            self._auto = True
            self._update_shift()
        else:
            self._auto = False
            self._shift = float(v)

    def _dist_sqr(self, args):
        if len(args) == 1:
            a = args[0]
            if isinstance(a, (tuple, list)) and len(a) == 3:
                return Real3D(a).sqr()
            return float(a) * float(a)
        return Real3D(*args).sqr()

    def computeEnergy(self, *args):
        ds = self._dist_sqr(args)
        if ds > self._cutoff * self._cutoff:
            return 0.0
        return self._energy_raw(ds) - self._shift

    def computeForce(self, *args):
        d = Real3D(args[0]) if len(args) == 1 else Real3D(*args)
        ds = d.sqr()
        if ds > self._cutoff * self._cutoff:
            return Real3D(0.0)
        return d * self._ffactor(ds)


class LennardJones(Potential):
    """interaction.LennardJones(epsilon=1.0, sigma=1.0, cutoff=inf, shift='auto')."""

    caprad = 0.0

    def __init__(self, epsilon=1.0, sigma=1.0, cutoff=infinity, shift="auto"):
        self._eps = float(epsilon)
        self._sig = float(sigma)
        Potential.__init__(self, cutoff, shift)

    epsilon = property(lambda s: s._eps, lambda s, v: s._set("_eps", v))
    sigma = property(lambda s: s._sig, lambda s, v: s._set("_sig", v))

    def _set(self, name, v):
        setattr(self, name, float(v))
        self._update_shift()

    def _energy_raw(self, ds):
        frac2 = self._sig * self._sig / ds
        frac6 = frac2 * frac2 * frac2
        return 4.0 * self._eps * (frac6 * frac6 - frac6)

    def _ffactor(self, ds):
        sig2 = self._sig * self._sig
        sig6 = sig2 * sig2 * sig2
        ff1 = 48.0 * self._eps * sig6 * sig6
        ff2 = 24.0 * self._eps * sig6
        frac2 = 1.0 / ds
        frac6 = frac2 * frac2 * frac2
        return frac6 * (ff1 * frac6 - ff2) * frac2


class LennardJonesCapped(LennardJones):
    """interaction.LennardJonesCapped(epsilon, sigma, cutoff, caprad, shift)
    (LennardJonesCapped.hpp:80-160): below caprad the force magnitude is frozen."""

    def __init__(self, epsilon=1.0, sigma=1.0, cutoff=infinity, caprad=0.0, shift="auto"):
        self._cap = float(caprad)
        LennardJones.__init__(self, epsilon, sigma, cutoff, shift)

    caprad = property(lambda s: s._cap, lambda s, v: s._set("_cap", v))

    def _energy_raw(self, ds):
        cs = self._cap * self._cap
        return LennardJones._energy_raw(self, cs if not ds > cs else ds)

    def _ffactor(self, ds):
        cs = self._cap * self._cap
        if ds > cs:
            return LennardJones._ffactor(self, ds)
        frac2 = (self._sig / self._cap) * (self._sig / self._cap)
        frac6 = frac2 * frac2 * frac2
        return 48.0 * self._eps * frac6 * (frac6 - 0.5) / (self._cap * math.sqrt(ds))


class FENE(Potential):
    """interaction.FENE(K=30.0, r0=0.0, rMax=1.5, cutoff=inf, shift=0.0)."""

    def __init__(self, K=30.0, r0=0.0, rMax=1.5, cutoff=infinity, shift=0.0):
        self._K = float(K)
        self._r0 = float(r0)
        self._rMax = float(rMax)
        Potential.__init__(self, cutoff, shift)

    K = property(lambda s: s._K, lambda s, v: s._set("_K", v))
    r0 = property(lambda s: s._r0, lambda s, v: s._set("_r0", v))
    rMax = property(lambda s: s._rMax, lambda s, v: s._set("_rMax", v))

    def _set(self, name, v):
        setattr(self, name, float(v))
        self._update_shift()

    def _energy_raw(self, ds):
        return -0.5 * (self._rMax * self._rMax) * self._K * math.log(
            1 - ((math.sqrt(ds) - self._r0) / self._rMax) ** 2)

    def _ffactor(self, ds):
        rms = self._rMax * self._rMax
        if self._r0 > ROUND_ERROR_PREC:
            r = math.sqrt(ds)
            return -self._K * (r - self._r0) / (r * (1 - ((r - self._r0) * (r - self._r0) / rms)))
        return -self._K / (1.0 - ds / rms)


class Interaction:
    """Interaction base (src/interaction/Interaction.hpp, Interaction.py:73-108)."""

    kind = None

    def __init__(self):
        self._system = None

    def _attach(self, system):
        self._system = system
        self._push()

    def _detach(self):
        self._system = None

    def _push(self):
        pass

    def _handle(self):
        st = self._system.storage if self._system is not None else None
        if st is None:
            raise RuntimeError("interaction is not added to a system with storage")
        return st

    def computeEnergy(self):
        st = self._handle()
        v = ctypes.c_double()
        call(st._lib, "espp_energy", st._h, self.kind, ctypes.byref(v))
        return v.value

    def computeVirial(self):
        st = self._handle()
        v = ctypes.c_double()
        call(st._lib, "espp_virial", st._h, self.kind, ctypes.byref(v))
        return v.value

    def computeVirialTensor(self):
        import numpy as np
        st = self._handle()
        w = np.zeros(6)
        call(st._lib, "espp_virial_tensor", st._h, self.kind, dptr(w))
        return Tensor(w)

    def bondType(self):
        return 2  # Pair

    def computeEnergyAA(self, *a):
        return 0.0

    def computeEnergyCG(self, *a):
        return 0.0


class VerletListLennardJones(Interaction):
    """interaction.VerletListLennardJones(vl) (LennardJones.py:733-760,
    VerletListInteractionTemplate.hpp:46-489)."""

    kind = _abi.IA_LJ
    _capped = False

    def __init__(self, vl):
        Interaction.__init__(self)
        self._vl = vl
        self._pots = {}

    def setPotential(self, type1, type2, potential):
        if self._capped != isinstance(potential, LennardJonesCapped):
            raise TypeError("potential type does not match the interaction")
        self._pots[(int(type1), int(type2))] = potential
        self._pots[(int(type2), int(type1))] = potential
        if self._system is not None:
            self._push()
            self._system.maxCutoff = max(self._system.maxCutoff, self.getMaxCutoff())

    def getPotential(self, type1, type2):
        return self._pots.get((int(type1), int(type2)))

    def getVerletList(self):
        return self._vl

    getVerletListLocal = getVerletList

    def getMaxCutoff(self):
        return max([p.cutoff for p in self._pots.values()] or [0.0])

    def _push(self):
        st = self._handle()
        if self._vl.system.storage is not st:
            raise RuntimeError("Verlet list belongs to another system")
        for (t1, t2), p in self._pots.items():
            if t1 > t2:
                continue
            call(st._lib, "espp_lj_set", st._h, t1, t2, p.epsilon, p.sigma, p.cutoff, p.shift,
                 p.caprad if self._capped else 0.0)


class VerletListLennardJonesCapped(VerletListLennardJones):
    """interaction.VerletListLennardJonesCapped(vl)."""

    _capped = True


class FixedPairListFENE(Interaction):
    """interaction.FixedPairListFENE(system, fpl, potential) (FENE.py:107-141,
    FixedPairListInteractionTemplate.hpp:46-623)."""

    kind = _abi.IA_FENE

    def __init__(self, system, vl, potential=None):
        Interaction.__init__(self)
        self._fpl = vl
        self._pot = potential
        self._pending_system = system

    def setPotential(self, potential):
        self._pot = potential
        if self._system is not None:
            self._push()

    def getPotential(self):
        return self._pot

    def setFixedPairList(self, fpl):
        self._fpl = fpl

    def getFixedPairList(self):
        return self._fpl

    def getMaxCutoff(self):
        return 0.0 if self._pot is None or math.isinf(self._pot.cutoff) else self._pot.cutoff

    def _push(self):
        st = self._handle()
        if self._pot is None:
            return
        p = self._pot
        call(st._lib, "espp_fene_set", st._h, p.K, p.r0, p.rMax, p.cutoff, p.shift)


class Tabulated(Potential):
    """interaction.Tabulated(itype, filename, cutoff=infinity) (Tabulated.py:610-615 and
    921-926, Tabulated.hpp:43-115, Tabulated.cpp:45-67): energy and force interpolated from a table
    file of (r, energy, force) lines; itype 1 linear, 2 Akima, 3 cubic spline.  The file is
    read and the table evaluated by the library, with the reference's parsing and
    interpolation arithmetic."""

    def __init__(self, itype, filename, cutoff=infinity):
        import numpy as np
        from ._lib import load_library
        self._lib = load_library()
        self._itype = int(itype)
        self._filename = str(filename)
        n = ctypes.c_int64()
        path = self._filename.encode()
        call(self._lib, "espp_tab_read", path, 0, None, None, None, ctypes.byref(n))
        self._r, self._e, self._f = np.zeros(n.value), np.zeros(n.value), np.zeros(n.value)
        call(self._lib, "espp_tab_read", path, n.value, dptr(self._r), dptr(self._e),
             dptr(self._f), ctypes.byref(n))
        Potential.__init__(self, cutoff, 0.0)

    @property
    def filename(self):
        return self._filename

    @property
    def itype(self):
        return self._itype

    def _eval(self, r, force):
        x = ctypes.c_double(r)
        out = ctypes.c_double()
        call(self._lib, "espp_tab_eval", self._itype, len(self._r), dptr(self._r),
             dptr(self._e), dptr(self._f), 1, ctypes.byref(x),
             None if force else ctypes.byref(out), ctypes.byref(out) if force else None)
        return out.value

    def _energy_raw(self, ds):
        return self._eval(math.sqrt(ds), False)

    def _ffactor(self, ds):
        r = math.sqrt(ds)
        return self._eval(r, True) / r

    def _table(self):
        return (self._itype, len(self._r), dptr(self._r), dptr(self._e), dptr(self._f))


class VerletListTabulated(Interaction):
    """interaction.VerletListTabulated(vl) (Tabulated.py:816-829, Tabulated.cpp:85-95)."""

    kind = _abi.IA_TAB_PAIR

    def __init__(self, vl):
        Interaction.__init__(self)
        self._vl = vl
        self._pots = {}

    def setPotential(self, type1, type2, potential):
        if not isinstance(potential, Tabulated):
            raise TypeError("potential type does not match the interaction")
        self._pots[(int(type1), int(type2))] = potential
        self._pots[(int(type2), int(type1))] = potential
        if self._system is not None:
            self._push()
            self._system.maxCutoff = max(self._system.maxCutoff, self.getMaxCutoff())

    def getPotential(self, type1, type2):
        return self._pots.get((int(type1), int(type2)))

    def getVerletList(self):
        return self._vl

    getVerletListLocal = getVerletList

    def getMaxCutoff(self):
        return max([p.cutoff for p in self._pots.values()] or [0.0])

    def _push(self):
        st = self._handle()
        if self._vl.system.storage is not st:
            raise RuntimeError("Verlet list belongs to another system")
        for (t1, t2), p in self._pots.items():
            if t1 > t2:
                continue
            call(st._lib, "espp_tab_pair_set", st._h, t1, t2, *p._table(), p.cutoff, p.shift)


class FixedPairListTabulated(Interaction):
    """interaction.FixedPairListTabulated(system, fpl, potential) (Tabulated.py:841-851,
    Tabulated.cpp:147-158)."""

    kind = _abi.IA_TAB_BOND

    def __init__(self, system, fpl, potential=None):
        Interaction.__init__(self)
        self._fpl = fpl
        self._pot = potential
        self._pending_system = system

    def setPotential(self, potential):
        self._pot = potential
        if self._system is not None:
            self._push()

    def getPotential(self):
        return self._pot

    def setFixedPairList(self, fpl):
        self._fpl = fpl

    def getFixedPairList(self):
        return self._fpl

    def getMaxCutoff(self):
        return 0.0 if self._pot is None or math.isinf(self._pot.cutoff) else self._pot.cutoff

    def _push(self):
        st = self._handle()
        if self._pot is None:
            return
        p = self._pot
        call(st._lib, "espp_tab_bond_set", st._h, *p._table(), p.cutoff, p.shift)


class Cosine:
    """interaction.Cosine(K=1.0, theta0=0.0) (Cosine.py:59-64, Cosine.hpp:38-125):
    E(theta) = K (1 + cos(theta - theta0))."""

    def __init__(self, K=1.0, theta0=0.0):
        self.K = float(K)
        self.theta0 = float(theta0)

    def computeEnergy(self, theta):
        return self.K * (1.0 + math.cos(float(theta) - self.theta0))

    def computeForce(self, theta):
        # AngularPotential computeForce(theta) of Cosine returns K (Cosine.hpp:121)
        return self.K


class FixedTripleListCosine(Interaction):
    """interaction.FixedTripleListCosine(system, ftl, potential) (Cosine.py:66-95,
    FixedTripleListInteractionTemplate.hpp:46-333)."""

    kind = _abi.IA_COSINE

    def __init__(self, system, ftl, potential=None):
        Interaction.__init__(self)
        self._ftl = ftl
        self._pot = potential
        self._pending_system = system

    def setPotential(self, potential):
        self._pot = potential
        if self._system is not None:
            self._push()

    def getPotential(self):
        return self._pot

    def getFixedTripleList(self):
        return self._ftl

    def getMaxCutoff(self):
        return 0.0

    def bondType(self):
        return 3  # Angular

    def _push(self):
        st = self._handle()
        if self._pot is not None:
            call(st._lib, "espp_cosine_set", st._h, self._pot.K, self._pot.theta0)


class TabulatedAngular(Tabulated):
    """interaction.TabulatedAngular(itype, filename, cutoff=infinity) (TabulatedAngular.py,
    TabulatedAngular.hpp:36-113, TabulatedAngular.cpp:40-64): E(theta) and f = -dE/dtheta
    interpolated from a table file of (theta, energy, force) lines; itype 1 linear, 2 Akima,
    3 cubic spline."""

    def computeEnergy(self, theta):
        return self._eval(float(theta), False)

    def computeForce(self, theta):
        return self._eval(float(theta), True)


class FixedTripleListTabulatedAngular(Interaction):
    """interaction.FixedTripleListTabulatedAngular(system, ftl, potential)
    (TabulatedAngular.cpp:82-88, FixedTripleListInteractionTemplate.hpp:46-333)."""

    kind = _abi.IA_TAB_ANGLE

    def __init__(self, system, ftl, potential=None):
        Interaction.__init__(self)
        self._ftl = ftl
        self._pot = potential
        self._pending_system = system

    def setPotential(self, potential):
        self._pot = potential
        if self._system is not None:
            self._push()

    def getPotential(self):
        return self._pot

    def setFixedTripleList(self, ftl):
        self._ftl = ftl

    def getFixedTripleList(self):
        return self._ftl

    def getMaxCutoff(self):
        return 0.0

    def bondType(self):
        return 3  # Angular

    def _push(self):
        st = self._handle()
        if self._pot is not None:
            call(st._lib, "espp_tab_angle_set", st._h, *self._pot._table())
