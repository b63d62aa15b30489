"""System, storage, boundary conditions and pair lists of the drop-in API.

Mirrors the Python classes of ESPResSo++ that sit in front of the short-range MD step
(src/System.py, src/storage/DomainDecomposition.py, src/bc/OrthorhombicBC.py,
src/esutil/RNG.py, src/VerletList.py, src/FixedPairList.py) on one process.  All
particle state lives on the GPU behind one C-ABI system handle that the storage
creates; the classes here keep configuration and forward to the handle.
"""
import ctypes
import json
import math
import os
import sys

import numpy as np

from . import _abi
from ._abi import call, dptr, i32ptr, i64ptr
from ._lib import load_library

infinity = float("inf")

_DEFAULT_PRECISION = os.environ.get("ESPP_B200_PRECISION", "fp64")


def set_default_precision(precision):
    """'fp64' (reference arithmetic, plain form) or 'mixed' (FP32 pair forces with int64
    fixed-point sums, FP64 integrator); used by storages created afterwards."""
    global _DEFAULT_PRECISION
    _precision_code(precision)
    _DEFAULT_PRECISION = precision


def _precision_code(p):
    if p in ("fp64", "double", _abi.PREC_FP64):
        return _abi.PREC_FP64
    if p in ("mixed", _abi.PREC_MIXED):
        return _abi.PREC_MIXED
    raise ValueError("precision must be 'fp64' or 'mixed', got %r" % (p,))


class Real3D(tuple):
    """3-vector of reals (src/Real3D.hpp)."""

    def __new__(cls, *args):
        if len(args) == 0:
            v = (0.0, 0.0, 0.0)
        elif len(args) == 1:
            a = args[0]
            v = (float(a),) * 3 if np.isscalar(a) else tuple(float(x) for x in a)
        else:
            v = tuple(float(x) for x in args)
        if len(v) != 3:
            raise TypeError("Real3D needs 3 components")
        return tuple.__new__(cls, v)

    x = property(lambda self: self[0])
    y = property(lambda self: self[1])
    z = property(lambda self: self[2])

    def __add__(self, o):
        return Real3D(self[0] + o[0], self[1] + o[1], self[2] + o[2])

    def __sub__(self, o):
        return Real3D(self[0] - o[0], self[1] - o[1], self[2] - o[2])

    def __mul__(self, o):
        if np.isscalar(o):
            return Real3D(self[0] * o, self[1] * o, self[2] * o)
        return self[0] * o[0] + self[1] * o[1] + self[2] * o[2]

    __rmul__ = __mul__

    def sqr(self):
        return self[0] * self[0] + self[1] * self[1] + self[2] * self[2]

    def abs(self):
        return math.sqrt(self.sqr())


class Int3D(tuple):
    """3-vector of ints (src/Int3D.hpp)."""

    def __new__(cls, *args):
        if len(args) == 0:
            v = (0, 0, 0)
        elif len(args) == 1:
            a = args[0]
            v = (int(a),) * 3 if np.isscalar(a) else tuple(int(x) for x in a)
        else:
            v = tuple(int(x) for x in args)
        if len(v) != 3:
            raise TypeError("Int3D needs 3 components")
        return tuple.__new__(cls, v)


class Tensor(tuple):
    """Symmetric tensor, components xx, yy, zz, xy, xz, yz (src/Tensor.hpp:125-133)."""

    def __new__(cls, *args):
        v = tuple(float(x) for x in (args[0] if len(args) == 1 else args))
        if len(v) != 6:
            raise TypeError("Tensor needs 6 components")
        return tuple.__new__(cls, v)


class RNG:
    """esutil.RNG(seed): uniform [0,1) draws on the host (src/esutil/RNG.cpp:40-66).
    The seed also keys the GPU Langevin noise of a system that uses this RNG."""

    def __init__(self, seed=12345):
        self.seed = int(seed)
        self._g = np.random.Generator(np.random.PCG64(self.seed))
        self._keyed = False  # a storage has keyed its Langevin noise on this seed

    def __call__(self, n=None):
        if n is None:
            return float(self._g.random())
        return int(self._g.integers(0, n))

    def uniform(self):
        return float(self._g.random())

    def normal(self):
        return float(self._g.normal())

    def get_seed(self):
        return self.seed

    def saveState(self, step):
        """Writes the generator state to the file "rng.<step>" in the working directory,
        one line per rank (RNG::saveState, src/esutil/RNG.cpp:86-108).  The line holds
        the seed, which keys the Langevin noise, and the host generator's state."""
        line = json.dumps({"seed": self.seed, "state": self._g.bit_generator.state})
        with open("rng." + str(int(step)), "w") as f:
            f.write(line + "\n")

    def loadState(self, fname):
        """Restores a state written by saveState (RNG::loadState, RNG.cpp:110-138).  As
        there, a file whose number of lines differs from the number of ranks (one) leaves
        the state unchanged with a warning.  The Langevin noise of a system is keyed on
        the seed it was created with, so a saved seed different from that key also leaves
        the state unchanged with a warning."""
        with open(fname) as f:
            lines = [ln for ln in f.read().split("\n") if ln]
        if len(lines) != 1:
            sys.stderr.write("# Warning: The number of processes does not match the number "
                             "of saved random number generators.\n"
                             "           The old states are not restored.\n")
            return
        saved = json.loads(lines[0])
        if self._keyed and int(saved["seed"]) != self.seed:
            sys.stderr.write("# Warning: the saved seed %d differs from seed %d, which keys "
                             "the Langevin noise of systems already created from this RNG.\n"
                             "           The old states are not restored.\n"
                             % (int(saved["seed"]), self.seed))
            return
        self.seed = int(saved["seed"])
        g = np.random.Generator(np.random.PCG64(self.seed))
        g.bit_generator.state = saved["state"]
        self._g = g


class OrthorhombicBC:
    """bc.OrthorhombicBC(rng, boxL) (src/bc/OrthorhombicBC.cpp:40-178)."""

    def __init__(self, rng, boxL):
        self.rng = rng
        self.boxL = boxL

    @property
    def boxL(self):
        return self._boxL

    @boxL.setter
    def boxL(self, v):
        self._boxL = Real3D(v)

    def getRandomPos(self):
        return Real3D(self._boxL[0] * self.rng(), self._boxL[1] * self.rng(),
                      self._boxL[2] * self.rng())

    def getMinimumImageVector(self, pos1, pos2):
        d = []
        for k in range(3):
            dk = pos1[k] - pos2[k]
            dk -= round(dk / self._boxL[k]) * self._boxL[k]
            d.append(dk)
        return Real3D(d)

    def getFoldedPosition(self, pos, imageBox=None):
        p = list(pos)
        img = list(imageBox) if imageBox is not None else [0, 0, 0]
        for k in range(3):
            t = int(math.floor(p[k] * (1.0 / self._boxL[k])))
            img[k] += t
            p[k] -= t * self._boxL[k]
        return Real3D(p), Int3D(img)

    def getUnfoldedPosition(self, pos, imageBox):
        return Real3D([pos[k] + imageBox[k] * self._boxL[k] for k in range(3)])


class System:
    """espressopp.System (src/System.cpp:40-105): holds bc, rng, skin, storage and the
    short-range interactions; maxCutoff is the largest interaction cutoff."""

    def __init__(self):
        self.rng = None
        self.bc = None
        self._skin = 0.0
        self._storage = None
        self.shortRangeInteractions = []
        self.maxCutoff = 0.0
        self._interaction2id = {}  # name -> index in shortRangeInteractions (System.py:134-192)
        self._integrator = None
        self._trace = False

    @property
    def integrator(self):
        return self._integrator

    @integrator.setter
    def integrator(self, integ):
        self._integrator = integ

    @property
    def skin(self):
        return self._skin

    @skin.setter
    def skin(self, v):
        self._skin = float(v)
        if self._storage is not None:
            call(self._storage._lib, "espp_set_skin", self._storage._h, self._skin)

    @property
    def storage(self):
        return self._storage

    @storage.setter
    def storage(self, st):
        self._storage = st

    def addInteraction(self, interaction, name=None):
        if name is not None and name in self._interaction2id:
            raise RuntimeError('Interaction with name {} already defined.'.format(name))
        kind = getattr(interaction, "kind", None)
        if kind is not None and any(getattr(ia, "kind", None) == kind
                                    for ia in self.shortRangeInteractions):
            # the device holds one parameter table per interaction kind, so a second one
            # would overwrite the first one's table
            raise RuntimeError("a system holds one interaction of each kind; {} is already "
                               "added".format(type(interaction).__name__))
        self.shortRangeInteractions.append(interaction)
        interaction._attach(self)
        self.maxCutoff = max(self.maxCutoff, interaction.getMaxCutoff())
        if name is not None:
            self._interaction2id[name] = len(self.shortRangeInteractions) - 1
        return True

    def removeInteraction(self, i):
        ia = self.shortRangeInteractions.pop(i)
        ia._detach()
        # names above the removed index move down by one; the removed one's name is dropped
        self._interaction2id = {k: (v if v < i else v - 1)
                                for k, v in self._interaction2id.items() if v != i}

    def removeInteractionByName(self, name):
        if name not in self._interaction2id:
            raise RuntimeError('Interaction {} not found'.format(name))
        self.removeInteraction(self._interaction2id[name])

    def getAllInteractions(self):
        return {k: self.getInteraction(v) for k, v in self._interaction2id.items()}

    def getInteractionByName(self, name):
        return self.getInteraction(self._interaction2id[name])

    def getNameOfInteraction(self, number):
        for name, iid in self._interaction2id.items():
            if iid == number:
                return name
        return None

    def setTrace(self, switch):
        """System::setTrace (tracing of the reference's C++ calls): kept as a flag; the GPU
        library has no trace output."""
        self._trace = bool(switch)

    def getInteraction(self, i):
        """System.py:167-176: an empty list and an index out of range are errors."""
        ni = len(self.shortRangeInteractions)
        if ni == 0:
            raise RuntimeError("interaction list of system is empty")
        if not 0 <= i < ni:
            raise RuntimeError("Interaction number %i does not exist" % i)
        return self.shortRangeInteractions[i]

    def getNumberOfInteractions(self):
        return len(self.shortRangeInteractions)

    def scaleVolume(self, *args):
        raise NotImplementedError("volume scaling is outside the GPU short-range MD step")


class Particle:
    """Read view of one particle (Storage.getParticle); values are fetched on access."""

    def __init__(self, storage, pid):
        self._st = storage
        self.id = int(pid)

    def _get(self):
        return self._st._fetch(np.array([self.id], np.int64))

    @property
    def pos(self):
        return Real3D(self._get()[0][0])

    @property
    def v(self):
        return Real3D(self._get()[1][0])

    @property
    def f(self):
        return Real3D(self._get()[2][0])

    @property
    def imageBox(self):
        return Int3D(self._get()[3][0])

    @property
    def type(self):
        return int(self._st._types.get(self.id, 0))

    @property
    def mass(self):
        return float(self._st._masses.get(self.id, 1.0))

    def isGhost(self):
        return False


class DomainDecomposition:
    """storage.DomainDecomposition(system, nodeGrid, cellGrid, halfCellInt)
    (src/storage/DomainDecomposition.py:84-130, DomainDecomposition.cpp:70-85).

    With nodeGrid (1,1,1) it creates one GPU system handle.  With more nodes (cellGrid is
    then one node's grid, as from tools.decomp.cellGrid) the box is cut into
    nodeGrid[0] * nodeGrid[1] * nodeGrid[2] slabs along z, one system per slab
    (espressopp_b200.domain): one slab per rank under torch.distributed, or all slabs in
    this process without it.  ``precision`` ('fp64' or 'mixed') selects the pair force
    arithmetic; it defaults to set_default_precision()."""

    def __init__(self, system, nodeGrid="auto", cellGrid="auto", halfCellInt="auto",
                 nocheck=False, precision=None):
        if system.bc is None:
            raise RuntimeError("system has no boundary conditions")
        ng = Int3D(1, 1, 1) if nodeGrid == "auto" else Int3D(nodeGrid)
        if min(ng) < 1:
            raise ValueError("invalid node grid %s" % (tuple(ng),))
        if halfCellInt == "auto":
            halfCellInt = 1
        halfCellInt = int(halfCellInt)
        if cellGrid == "auto":
            cellGrid = Int3D(2, 2, 2)
        cellGrid = list(Int3D(cellGrid))
        for k in range(3):
            # one node: a 1-cell dimension takes 2 cells; with several nodes the whole box
            # has cellGrid x nodeGrid cells and the node's grid stays as given
            if cellGrid[k] == 1 and ng[k] == 1:
                cellGrid[k] = 2
        self.system = system
        self._cellGrid = Int3D(cellGrid)
        self._nodeGrid = ng
        self._lib = load_library()
        self._h = ctypes.c_void_p()
        prec = _precision_code(precision if precision is not None else _DEFAULT_PRECISION)
        self.precision = prec
        box = np.ascontiguousarray(system.bc.boxL, np.float64)
        seed = system.rng.get_seed() if system.rng is not None else 12345
        if system.rng is not None:
            system.rng._keyed = True
        self.halfCellInt = halfCellInt
        nodes = ng[0] * ng[1] * ng[2]
        if nodes > 1:
            # cellGrid is the grid of one node (DomainDecomposition.cpp:87-170): the whole
            # box has cellGrid x nodeGrid cells, cut here into `nodes` slabs along z, one
            # system per slab (espressopp_b200.domain)
            from . import domain
            from ._decomposed import DecomposedLibrary
            comm = domain.LocalComm()
            try:
                import torch.distributed as dist
                if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
                    comm = domain.TorchComm(dist)
            except ImportError:
                pass
            full = [self._cellGrid[k] * ng[k] for k in range(3)]
            self._sd = domain.SpatialDecomposition(
                box, float(system.skin), full, nodes, precision=prec,
                seed=int(seed) & 0xFFFFFFFFFFFFFFFF, comm=comm, lib=self._lib,
                half_cell_int=halfCellInt)
            self._lib = DecomposedLibrary(self._sd)
            self._h = ctypes.c_void_p(1)  # stands for the decomposition in mirror calls
        else:
            cg = np.ascontiguousarray(self._cellGrid, np.int32)
            call(self._lib, "espp_system_create", dptr(box), float(system.skin), i32ptr(cg),
                 prec, int(seed) & 0xFFFFFFFFFFFFFFFF, ctypes.byref(self._h))
            if halfCellInt != 1:
                call(self._lib, "espp_set_half_cell_int", self._h, halfCellInt)
        self._types = {}
        self._masses = {}
        self.next_id = 0

    def __del__(self):
        try:
            if self._h:
                self._lib.espp_system_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass

    # -- particles --------------------------------------------------------------------
    def addParticles(self, particleList, *properties):
        """Storage.addParticles (src/storage/Storage.py:233-330).  Known properties: id,
        type, mass, pos, v; other per-particle properties are accepted and ignored."""
        if len(particleList) == 0:
            return
        props = list(properties) if properties else ["id", "pos"]
        if "id" not in props or "pos" not in props:
            raise ValueError("particle properties must include 'id' and 'pos'")
        n = len(particleList)
        ids = np.empty(n, np.int64)
        pos = np.empty((n, 3))
        vel = np.zeros((n, 3))
        typ = np.zeros(n, np.int32)
        mass = np.ones(n)
        col = {p: k for k, p in enumerate(props)}
        for r, part in enumerate(particleList):
            ids[r] = int(part[col["id"]])
            pos[r] = tuple(part[col["pos"]])
            if "v" in col:
                vel[r] = tuple(part[col["v"]])
            if "type" in col:
                typ[r] = int(part[col["type"]])
            if "mass" in col:
                mass[r] = float(part[col["mass"]])
        call(self._lib, "espp_add_particles", self._h, n, i64ptr(ids), i32ptr(typ),
             dptr(mass), dptr(pos.reshape(-1)), dptr(vel.reshape(-1)))
        for k in range(n):
            self._types[int(ids[k])] = int(typ[k])
            self._masses[int(ids[k])] = float(mass[k])
        self.next_id = max(self.next_id, int(ids.max()) + 1)

    def addParticle(self, pid, pos):
        self.addParticles([[pid, Real3D(pos)]], "id", "pos")

    def decompose(self):
        call(self._lib, "espp_decompose", self._h)

    def getParticle(self, pid):
        if int(pid) not in self._types:
            return None
        return Particle(self, pid)

    def particleExists(self, pid):
        return int(pid) in self._types

    def getRealParticleIDs(self):
        return sorted(self._types)

    def getNRealParticles(self):
        return len(self._types)

    def modifyParticle(self, pid, prop, value):
        """Storage.modifyParticle (src/storage/Storage.py:374-400) for 'pos', 'v' and
        'img'.  As there, a new position is taken as unfolded: the image is reset."""
        ids = np.array([int(pid)], np.int64)
        prop = prop.lower()
        if prop not in ("pos", "v", "img"):
            raise ValueError("only 'pos', 'v' and 'img' can be modified on the GPU storage")
        if prop == "img":
            img = np.ascontiguousarray(tuple(value), np.int32)
            call(self._lib, "espp_set_images", self._h, 1, i64ptr(ids), i32ptr(img))
            return
        v = np.ascontiguousarray(tuple(value), np.float64)
        if prop == "pos":
            call(self._lib, "espp_set_particles", self._h, 1, i64ptr(ids), dptr(v), None)
            zero = np.zeros(3, np.int32)
            call(self._lib, "espp_set_images", self._h, 1, i64ptr(ids), i32ptr(zero))
        else:
            call(self._lib, "espp_set_particles", self._h, 1, i64ptr(ids), None, dptr(v))

    def getCellGrid(self):
        return self._cellGrid

    def getNodeGrid(self):
        return self._nodeGrid

    def _fetch(self, ids):
        n = len(ids)
        pos = np.zeros((n, 3))
        vel = np.zeros((n, 3))
        frc = np.zeros((n, 3))
        img = np.zeros((n, 3), np.int32)
        call(self._lib, "espp_get_particles", self._h, n, i64ptr(ids), dptr(pos), dptr(vel),
             dptr(frc), i32ptr(img))
        return pos, vel, frc, img

    def getAll(self):
        """(ids, pos, v, f, imageBox) arrays of all particles, sorted by id."""
        ids = np.array(sorted(self._types), np.int64)
        pos, vel, frc, img = self._fetch(ids)
        return ids, pos, vel, frc, img

    def setVelocities(self, ids, vel):
        ids = np.ascontiguousarray(ids, np.int64)
        v = np.ascontiguousarray(vel, np.float64).reshape(-1)
        call(self._lib, "espp_set_particles", self._h, len(ids), i64ptr(ids), None, dptr(v))

    def setImages(self, ids, img):
        """Image counts of many particles at once (modifyParticle(pid, 'img', ...) for
        each), e.g. to restore a checkpoint written from getAll()."""
        ids = np.ascontiguousarray(ids, np.int64)
        im = np.ascontiguousarray(img, np.int32).reshape(-1)
        call(self._lib, "espp_set_images", self._h, len(ids), i64ptr(ids), i32ptr(im))

    _ARRAY_PROPS = ("id", "posx", "posy", "posz", "vx", "vy", "vz", "type", "mass")

    def addParticlesArray(self, particleList, *properties):
        """Storage.addParticlesArray (src/storage/Storage.py:432-535): particles as the
        rows of a 2-d array whose columns the properties name (default id, posx, posy,
        posz); id and the three position columns are mandatory.  Columns of properties the
        GPU storage does not hold (modepos, f, q, radius, AdResS, ...) are accepted and
        ignored; an unknown name is a SyntaxError, as there."""
        known = set(self._ARRAY_PROPS) | {
            "modeposx", "modeposy", "modeposz", "modemomx", "modemomy", "modemomz", "fx",
            "fy", "fz", "fmx", "fmy", "fmz", "q", "radius", "fradius", "vradius", "varmass",
            "adrat", "lambda_adr", "lambda_adrd", "state", "pib"}
        props = [p.lower() for p in properties] if properties else ["id", "posx", "posy",
                                                                     "posz"]
        for p in props:
            if p not in known:
                raise SyntaxError("unknown particle property: %s" % p)
        col = {p: k for k, p in enumerate(props)}
        for p in ("id", "posx", "posy", "posz"):
            if p not in col:
                raise AssertionError("particle property %s is mandatory" % p)
        for trio in (("vx", "vy", "vz"), ("fx", "fy", "fz"), ("modeposx", "modeposy",
                     "modeposz"), ("modemomx", "modemomy", "modemomz"), ("fmx", "fmy", "fmz")):
            if len({t in col for t in trio}) != 1:
                raise AssertionError("Missing at least one of the 3d coordinates of property "
                                     "\"%s\"" % trio[0][:-1])
        arr = np.asarray(particleList, np.float64)
        if arr.size == 0:
            return
        arr = arr.reshape(len(arr), -1)
        names = ["id", "pos"]
        rows = [[int(r[col["id"]]), Real3D(r[col["posx"]], r[col["posy"]], r[col["posz"]])]
                for r in arr]
        if "vx" in col:
            names.append("v")
            for row, r in zip(rows, arr):
                row.append(Real3D(r[col["vx"]], r[col["vy"]], r[col["vz"]]))
        for p in ("type", "mass"):
            if p in col:
                names.append(p)
                for row, r in zip(rows, arr):
                    row.append(int(r[col[p]]) if p == "type" else float(r[col[p]]))
        self.addParticles(rows, *names)

    def _reload(self, keep):
        """Replaces the particle set by the particles with the given ids, state kept;
        the next step re-sorts them."""
        ids = np.array(sorted(keep), np.int64)
        pos, vel, _, img = self._fetch(ids) if len(ids) else (np.zeros((0, 3)),) * 2 + (
            None, np.zeros((0, 3), np.int32))
        typ = np.array([self._types[int(i)] for i in ids], np.int32)
        mass = np.array([self._masses[int(i)] for i in ids], np.float64)
        call(self._lib, "espp_dd_load", self._h, len(ids), i64ptr(ids), i32ptr(typ),
             dptr(mass), dptr(np.ascontiguousarray(pos)), dptr(np.ascontiguousarray(vel)),
             i32ptr(np.ascontiguousarray(img, np.int32)), None)
        self._types = {int(i): self._types[int(i)] for i in ids}
        self._masses = {int(i): self._masses[int(i)] for i in ids}

    def removeParticle(self, pid):
        """Storage::removeParticle (src/storage/Storage.cpp:315-348): 1 if the particle
        existed and was removed, else 0.  Bonds and triples of a removed particle must be
        removed by the caller, as in the reference."""
        pid = int(pid)
        if pid not in self._types:
            return 0
        self._reload([i for i in self._types if i != pid])
        return 1

    def removeAllParticles(self):
        """Storage::removeAllParticles (src/storage/Storage.cpp:350-358)."""
        self._reload([])

    def savePositions(self, idList):
        """Storage::savePosition for each id (src/storage/Storage.cpp:804-829): position
        and image of each existing particle, restored by restorePositions."""
        ids = np.array([int(i) for i in idList if int(i) in self._types], np.int64)
        if not hasattr(self, "_saved"):
            self._saved = {}
        if len(ids):
            pos, _, _, img = self._fetch(ids)
            for k, i in enumerate(ids):
                self._saved[int(i)] = (pos[k].copy(), img[k].copy())

    def restorePositions(self):
        """Storage::restorePositions (src/storage/Storage.cpp:830-869)."""
        saved = getattr(self, "_saved", {})
        if not saved:
            raise RuntimeError(" There is nothing to restore. Check whether you saved positions")
        ids = np.array([i for i in saved if i in self._types], np.int64)
        if len(ids):
            pos = np.ascontiguousarray([saved[int(i)][0] for i in ids], np.float64)
            img = np.ascontiguousarray([saved[int(i)][1] for i in ids], np.int32)
            call(self._lib, "espp_set_particles", self._h, len(ids), i64ptr(ids),
                 dptr(pos.reshape(-1)), None)
            call(self._lib, "espp_set_images", self._h, len(ids), i64ptr(ids),
                 i32ptr(img.reshape(-1)))

    def clearSavedPositions(self):
        self._saved = {}

    def printRealParticles(self):
        """Storage.printRealParticles (src/storage/Storage.py:426-430): one line per
        particle, with rank 0 as the CPU column."""
        ids = np.array(self.getRealParticleIDs(), np.int64)
        if len(ids) == 0:
            return
        pos = self._fetch(ids)[0]
        for k, pid in enumerate(ids):
            sys.stdout.write("CPU %-3i ID %-5i TYPE %-3i POS(%8.3f, %8.3f, %8.3f)\n" % (
                0, pid, self._types[int(pid)], pos[k][0], pos[k][1], pos[k][2]))


class VerletList:
    """VerletList(system, cutoff, exclusionlist=[], useBuffers=True, useSOA=False)
    (src/VerletList.py:66-126, src/VerletList.cpp:196-536).  ``useBuffers`` and
    ``useSOA`` select CPU code paths in the reference and do not change the pair set;
    they are accepted and ignored."""

    def __init__(self, system, cutoff, exclusionlist=[], useBuffers=True, useSOA=False):
        if system.storage is None:
            raise RuntimeError("system has no storage")
        self.system = system
        self.cutoff = float(cutoff)
        st = system.storage
        ex = np.ascontiguousarray(list(exclusionlist), np.int64).reshape(-1)
        call(st._lib, "espp_vl_create", st._h, self.cutoff, len(ex) // 2,
             i64ptr(ex) if len(ex) else None)
        self._connected = True

    @property
    def _st(self):
        return self.system.storage

    @property
    def builds(self):
        v = ctypes.c_int64()
        call(self._st._lib, "espp_vl_builds", self._st._h, ctypes.byref(v))
        return v.value

    def totalSize(self):
        v = ctypes.c_int64()
        call(self._st._lib, "espp_vl_size", self._st._h, ctypes.byref(v))
        return v.value

    localSize = totalSize

    def exclude(self, exclusionlist):
        ex = np.ascontiguousarray(list(exclusionlist), np.int64).reshape(-1)
        call(self._st._lib, "espp_vl_create", self._st._h, self.cutoff, len(ex) // 2,
             i64ptr(ex) if len(ex) else None)

    def rebuild(self):
        call(self._st._lib, "espp_vl_rebuild", self._st._h)

    def pairs(self):
        """All pairs as an (n, 2) int64 array of (smaller id, larger id), sorted."""
        n = self.totalSize()
        out = np.zeros((max(n, 1), 2), np.int64)
        got = ctypes.c_int64()
        call(self._st._lib, "espp_vl_pairs", self._st._h, n, i64ptr(out), ctypes.byref(got))
        return out[: got.value]

    def getAllPairs(self):
        """Like the reference's PMI proxy: one list of (id1, id2) tuples per worker."""
        return [[(int(a), int(b)) for a, b in self.pairs()]]

    def getVerletCutoff(self):
        return self.cutoff + self.system.skin

    def connect(self):
        self._connected = True

    def disconnect(self):
        self._connected = False

    def resetTimers(self):
        pass

    def getTimers(self):
        return [(0.0,)]


class FixedPairList:
    """FixedPairList(storage) (src/FixedPairList.py:60-148, FixedPairList.cpp:88-315)."""

    def __init__(self, storage):
        self.storage = storage
        self._bonds = []

    def add(self, pid1, pid2):
        self.addBonds([(pid1, pid2)])
        return True

    def addBonds(self, bondlist):
        b = np.ascontiguousarray([(int(a), int(c)) for a, c in bondlist], np.int64).reshape(-1)
        if len(b) == 0:
            return
        call(self.storage._lib, "espp_bonds_add", self.storage._h, len(b) // 2, i64ptr(b))
        self._bonds.extend((min(int(a), int(c)), max(int(a), int(c))) for a, c in bondlist)

    def getBonds(self):
        return [list(self._bonds)]

    def size(self):
        return len(self._bonds)

    totalSize = size

    def getAllBonds(self):
        """FixedPairList::getAllBonds (FixedPairList.cpp:167-200): every bond as a
        (pid1, pid2) tuple, pid1 < pid2."""
        return list(self._bonds)

    def remove(self):
        """FixedPairList::remove (FixedPairList.cpp:317-324): empties the list."""
        call(self.storage._lib, "espp_bonds_clear", self.storage._h)
        self._bonds = []

    def getLongtimeMaxBondSqr(self):
        """The longest bond^2 seen by any force pass since the last reset
        (FixedPairListInteractionTemplate.hpp:145-150)."""
        v = ctypes.c_double()
        call(self.storage._lib, "espp_bonds_max_sqr", self.storage._h, ctypes.byref(v))
        return v.value

    def resetLongtimeMaxBond(self):
        call(self.storage._lib, "espp_bonds_reset_max", self.storage._h)

    def getLongtimeMaxBondLocal(self):
        """One value per worker, as the reference's pmiinvoke returns it."""
        return [math.sqrt(self.getLongtimeMaxBondSqr())]

    def getLongtimeMaxBond(self):
        return max(self.getLongtimeMaxBondLocal())


class FixedTripleList:
    """FixedTripleList(storage) (src/FixedTripleList.py:60-125): angle triples (pid1, pid2,
    pid3) with pid2 the centre."""

    def __init__(self, storage):
        self.storage = storage
        self._triples = []

    def add(self, pid1, pid2, pid3):
        self.addTriples([(pid1, pid2, pid3)])
        return True

    def addTriples(self, triplelist):
        t = np.ascontiguousarray([(int(a), int(b), int(c)) for a, b, c in triplelist],
                                 np.int64).reshape(-1)
        if len(t) == 0:
            return
        call(self.storage._lib, "espp_triples_add", self.storage._h, len(t) // 3, i64ptr(t))
        self._triples.extend((int(a), int(b), int(c)) for a, b, c in triplelist)

    def getTriples(self):
        return [list(self._triples)]

    def remove(self):
        """FixedTripleList.remove (FixedTripleList.py:97-100): empties the list."""
        call(self.storage._lib, "espp_triples_clear", self.storage._h)
        self._triples = []

    def size(self):
        return len(self._triples)

    totalSize = size
