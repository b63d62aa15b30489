"""Test-side driver of the C ABI (include/espp_b200.h).

``Sim(lib, ...)`` issues the same sequence of ABI calls on whichever library it is
given: the CUDA library (espressopp_b200.load_library()) or the CPU oracle
(``oracle_lib()``).  Parity tests build two ``Sim``s on identical inputs and compare.
The oracle is test infrastructure: only tests, smoke() and bench.py's CPU-baseline leg
load it.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

from espressopp_b200 import _abi
from espressopp_b200._abi import call, dptr, i32ptr, i64ptr

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(REPO, "oracle", "_build", "liboracle_espp.so")
GOLDEN = os.path.join(REPO, "tests", "golden")

_oracle = None


def oracle_lib():
    """Loads (building if needed) the FP64 CPU oracle library."""
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "oracle")])
        lib = ctypes.CDLL(ORACLE_SO)
        D = ctypes.POINTER(ctypes.c_double)
        U = ctypes.POINTER(ctypes.c_uint32)
        _abi.bind(lib, extra={
            "espp_oracle_philox": (ctypes.c_int32, [U, U, U]),
            "espp_oracle_lj_eval": (ctypes.c_int32, [ctypes.c_double] * 5 + [D, D, D]),
            "espp_oracle_fene_eval": (ctypes.c_int32, [ctypes.c_double] * 5 + [D, D, D]),
            "espp_vec_run": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int64]),
            "espp_vec_pairs": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int64,
                                                ctypes.POINTER(ctypes.c_int64),
                                                ctypes.POINTER(ctypes.c_int64)]),
        })
        _oracle = lib
    return _oracle


def cuda_lib():
    import espressopp_b200
    return espressopp_b200.load_library()


class Sim:
    def __init__(self, lib, box, skin, cell_grid, precision=_abi.PREC_FP64, seed=12345,
                 half_cell_int=1):
        self.lib = lib
        self.h = ctypes.c_void_p()
        b = np.ascontiguousarray(box, np.float64)
        cg = np.ascontiguousarray(cell_grid, np.int32)
        call(lib, "espp_system_create", dptr(b), float(skin), i32ptr(cg), int(precision),
             int(seed), ctypes.byref(self.h))
        if half_cell_int != 1:
            call(lib, "espp_set_half_cell_int", self.h, int(half_cell_int))

    def __del__(self):
        try:
            if self.h:
                self.lib.espp_system_destroy(self.h)
                self.h = ctypes.c_void_p()
        except Exception:
            pass

    def add(self, ids, pos, vel=None, types=None, mass=None):
        ids = np.ascontiguousarray(ids, np.int64)
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float64).reshape(-1)
        types = None if types is None else np.ascontiguousarray(types, np.int32)
        mass = None if mass is None else np.ascontiguousarray(mass, np.float64)
        call(self.lib, "espp_add_particles", self.h, len(ids), i64ptr(ids), i32ptr(types),
             dptr(mass), dptr(pos), dptr(vel))
        return self

    def decompose(self):
        call(self.lib, "espp_decompose", self.h)

    def vl(self, cutoff, excl=None):
        ex = None if excl is None else np.ascontiguousarray(excl, np.int64).reshape(-1)
        call(self.lib, "espp_vl_create", self.h, float(cutoff),
             0 if ex is None else len(ex) // 2, i64ptr(ex))

    def vl_rebuild(self):
        call(self.lib, "espp_vl_rebuild", self.h)

    def lj(self, t1, t2, eps, sig, rc, shift, caprad=0.0):
        call(self.lib, "espp_lj_set", self.h, t1, t2, eps, sig, rc, shift, caprad)

    def bonds(self, pairs):
        p = np.ascontiguousarray(pairs, np.int64).reshape(-1)
        call(self.lib, "espp_bonds_add", self.h, len(p) // 2, i64ptr(p))

    def fene(self, K=30.0, r0=0.0, rmax=1.5, rc=math.inf, shift=0.0):
        call(self.lib, "espp_fene_set", self.h, K, r0, rmax, rc, shift)

    def triples(self, trip):
        t = np.ascontiguousarray(trip, np.int64).reshape(-1)
        call(self.lib, "espp_triples_add", self.h, len(t) // 3, i64ptr(t))

    def cosine(self, K=1.5, theta0=3.1415926):
        call(self.lib, "espp_cosine_set", self.h, K, theta0)

    def tab_angle(self, itype, theta, e, f):
        th, ee, ff = (np.ascontiguousarray(a, np.float64) for a in (theta, e, f))
        call(self.lib, "espp_tab_angle_set", self.h, int(itype), len(th), dptr(th), dptr(ee),
             dptr(ff))

    def integrator(self, dt):
        call(self.lib, "espp_integrator_set", self.h, float(dt))

    def langevin(self, gamma, temperature, excl=None, enabled=True):
        ex = None if excl is None else np.ascontiguousarray(excl, np.int64)
        call(self.lib, "espp_langevin_set", self.h, 1 if enabled else 0, float(gamma),
             float(temperature), 0 if ex is None else len(ex), i64ptr(ex))

    def capforce(self, mode, cap):
        c = np.ascontiguousarray(np.broadcast_to(np.asarray(cap, np.float64), (3,)))
        call(self.lib, "espp_capforce_set", self.h, int(mode), dptr(c))

    def run(self, n):
        call(self.lib, "espp_run", self.h, int(n))

    def step(self):
        v = ctypes.c_int64()
        call(self.lib, "espp_step_get", self.h, ctypes.byref(v))
        return v.value

    def num_resorts(self):
        v = ctypes.c_int64()
        call(self.lib, "espp_num_resorts", self.h, ctypes.byref(v))
        return v.value

    def builds(self):
        v = ctypes.c_int64()
        call(self.lib, "espp_vl_builds", self.h, ctypes.byref(v))
        return v.value

    def energy(self, which):
        v = ctypes.c_double()
        call(self.lib, "espp_energy", self.h, which, ctypes.byref(v))
        return v.value

    def virial(self, which):
        v = ctypes.c_double()
        call(self.lib, "espp_virial", self.h, which, ctypes.byref(v))
        return v.value

    def virial_tensor(self, which):
        w = np.zeros(6)
        call(self.lib, "espp_virial_tensor", self.h, which, dptr(w))
        return w

    def kinetic(self):
        v = ctypes.c_double()
        n = ctypes.c_int64()
        call(self.lib, "espp_kinetic", self.h, ctypes.byref(v), ctypes.byref(n))
        return v.value, n.value

    def particles(self, ids):
        ids = np.ascontiguousarray(ids, np.int64)
        n = len(ids)
        pos = np.zeros((n, 3))
        vel = np.zeros((n, 3))
        frc = np.zeros((n, 3))
        img = np.zeros((n, 3), np.int32)
        call(self.lib, "espp_get_particles", self.h, n, i64ptr(ids), dptr(pos), dptr(vel),
             dptr(frc), i32ptr(img))
        return pos, vel, frc, img

    def vl_size(self):
        v = ctypes.c_int64()
        call(self.lib, "espp_vl_size", self.h, ctypes.byref(v))
        return v.value

    def pairs(self):
        n = self.vl_size()
        out = np.zeros((max(n, 1), 2), np.int64)
        got = ctypes.c_int64()
        call(self.lib, "espp_vl_pairs", self.h, n, i64ptr(out), ctypes.byref(got))
        return out[:got.value]

    def digest(self):
        out = (ctypes.c_uint64 * 4)()
        call(self.lib, "espp_vl_digest", self.h, out)
        return tuple(int(v) for v in out)

    def confs(self, key, ids):
        ids = np.ascontiguousarray(ids, np.int64)
        h = ctypes.c_void_p()
        call(self.lib, "espp_confs_create", self.h, int(key), len(ids), i64ptr(ids),
             ctypes.byref(h))
        return Confs(self.lib, h, len(ids))


class Confs:
    """Snapshot list (espp_confs_*) of one system, for the MSD tests."""

    def __init__(self, lib, h, n):
        self.lib, self.h, self.n = lib, h, n

    def __del__(self):
        try:
            if self.h:
                self.lib.espp_confs_destroy(self.h)
                self.h = ctypes.c_void_p()
        except Exception:
            pass

    def gather(self):
        call(self.lib, "espp_confs_gather", self.h)

    def push(self, xyz):
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1)
        call(self.lib, "espp_confs_push", self.h, dptr(xyz))

    def size(self):
        m = ctypes.c_int32()
        call(self.lib, "espp_confs_size", self.h, ctypes.byref(m))
        return m.value

    def get(self, m):
        out = np.zeros((self.n, 3))
        call(self.lib, "espp_confs_get", self.h, int(m), dptr(out))
        return out

    def msd(self):
        out = np.zeros(self.size())
        call(self.lib, "espp_msd", self.h, dptr(out))
        return out

    def msd_chain(self, chainlength):
        out = np.zeros(self.size())
        call(self.lib, "espp_msd_chain_com", self.h, int(chainlength), dptr(out))
        return out


def _mix64(z):
    z = (z + np.uint64(0x9E3779B97F4A7C15))
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def pair_digest(pairs):
    """espp_vl_digest of an (n, 2) array of id pairs, computed with numpy."""
    p = np.asarray(pairs, np.int64).reshape(-1, 2)
    lo = np.minimum(p[:, 0], p[:, 1]).astype(np.uint64)
    hi = np.maximum(p[:, 0], p[:, 1]).astype(np.uint64)
    with np.errstate(over="ignore"):
        h = _mix64(_mix64(lo) ^ hi)
        s1 = int(np.sum(h, dtype=np.uint64))
        s2 = int(np.sum(_mix64(h), dtype=np.uint64))
    x = int(np.bitwise_xor.reduce(h)) if len(h) else 0
    return (len(p), s1, x, s2)


def cosine_angle_table(K=1.5, theta0=3.1415926, n=4001):
    """E(theta) = K (1 + cos(theta - theta0)) and f = -dE/dtheta on [0, pi]."""
    th = np.linspace(0.0, math.pi, n)
    return th, K * (1.0 + np.cos(th - theta0)), K * np.sin(th - theta0)


def msd_reference(snaps):
    """MeanSquareDispl::compute (MeanSquareDispl.cpp:89-137) on snapshots (M, N, 3)."""
    M, N = snaps.shape[0], snaps.shape[1]
    out = np.zeros(M)
    for m in range(M):
        z = sum(np.sum((snaps[t] - snaps[t + m]) ** 2) for t in range(M - m))
        out[m] = z / (M - m) / (6.0 * N)
    return out


def msd_chain_reference(snaps, chainlength):
    """MeanSquareDispl::computeG3 (MeanSquareDispl.cpp:312-425) on snapshots (M, N, 3)."""
    M, N = snaps.shape[0], snaps.shape[1]
    nch = N // chainlength
    com = snaps[:, :nch * chainlength].reshape(M, nch, chainlength, 3).mean(axis=2)
    rel = com - com.mean(axis=1, keepdims=True)
    out = np.zeros(M)
    for m in range(M):
        z = sum(np.sum((rel[t] - rel[t + m]) ** 2) for t in range(M - m))
        out[m] = z / (6.0 * nch) / (M - m)
    return out


def cell_grid(box, rc, skin, half_cell_int=1):
    """tools.decomp.cellGrid (src/tools/decomp.py:322-342) for nodeGrid (1,1,1)."""
    return [int((b * half_cell_int) / (rc + skin)) for b in box]


def load_lj2048():
    z = np.load(os.path.join(GOLDEN, "lj_fluid_2048.npz"))
    return z["pid"], z["pos"], z["vel"], z["box"]


def load_polymer40k(angles=False):
    import json
    z = np.load(os.path.join(GOLDEN, "polymer_melt_40k.npz"))
    pos = z["pos_milli"].astype(np.float64) / 1000.0
    with open(os.path.join(GOLDEN, "polymer_melt_40k.json")) as f:
        gold = json.load(f)
    if angles:
        return pos, z["bonds"].astype(np.int64), z["box"], gold, z["angles"].astype(np.int64)
    return pos, z["bonds"].astype(np.int64), z["box"], gold


def lattice(n_side, rho, jitter, seed):
    """Simple-cubic lattice with uniform jitter (tools/lattice.py:24-71 layout)."""
    N = n_side ** 3
    L = (N / rho) ** (1.0 / 3.0)
    a = L / n_side
    g = np.arange(n_side)
    i, j, k = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([0.5 * a + i * a, 0.5 * a + j * a, 0.5 * a + k * a], -1).reshape(-1, 3)
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = pos + rng.uniform(-jitter, jitter, size=pos.shape)
    return pos, np.array([L, L, L])


def mb_velocities(N, T, seed):
    """Maxwell-Boltzmann velocities, rescaled to T and zero net momentum
    (tools/velocities.py:27-95)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    v = rng.normal(0.0, math.sqrt(T), size=(N, 3))
    ek = 0.5 * np.sum(v * v)
    v *= math.sqrt(T / (2.0 * ek / (3 * N)))
    v -= v.mean(axis=0)
    return v


def write_tab_file(pot, path, N, low, high, body=2):
    """Table file as testsuite/tabulated/polymer_melt_tabulated.py writeTabFile writes it:
    N equidistant r in [low, high], one "%15.8g %15.8g %15.8g" line (r, energy, force)."""
    delta = (high - low) / (N - 1)
    with open(path, "w") as out:
        for i in range(N):
            r = low + i * delta
            energy = pot.computeEnergy(r)
            force = pot.computeForce((r, 0.0, 0.0))[0]
            out.write("%15.8g %15.8g %15.8g\n" % (r, energy, force))


def read_tab(lib, path):
    """(r, e, f) arrays of a table file read through espp_tab_read of lib."""
    n = ctypes.c_int64()
    call(lib, "espp_tab_read", path.encode(), 0, None, None, None, ctypes.byref(n))
    r, e, f = np.zeros(n.value), np.zeros(n.value), np.zeros(n.value)
    call(lib, "espp_tab_read", path.encode(), n.value, dptr(r), dptr(e), dptr(f),
         ctypes.byref(n))
    return r, e, f


def polymer_tab_tables(tmpdir, lib):
    """The Akima tables of testsuite/tabulated/polymer_melt_tabulated.py (LJ eps=sig=1
    rc=1.12 shift 0 on [0.01, 1.12]; FENE K=30 r0=0 rMax=1.5 on [0.0001, 1.49]; N=257)."""
    from espressopp_b200 import interaction
    lj = interaction.LennardJones(epsilon=1.0, sigma=1.0, shift=False, cutoff=1.12)
    fene = interaction.FENE(K=30.0, r0=0.0, rMax=1.5)
    plj = os.path.join(str(tmpdir), "pot-lj.txt")
    pfene = os.path.join(str(tmpdir), "pot-fene.txt")
    write_tab_file(lj, plj, N=257, low=0.01, high=lj.cutoff)
    write_tab_file(fene, pfene, N=257, low=0.0001, high=1.49)
    return read_tab(lib, plj), read_tab(lib, pfene), plj, pfene
