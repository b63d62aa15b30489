"""Coarse-graining workflow for the learned potential: a fine-grained Kremer-Grest melt
is mapped 4 consecutive beads -> 1 site (centre of mass; mapped force = sum of the bead
forces), the bonded part is a Boltzmann-inverted bond table (FixedPairListTabulated), the
non-bonded part a learned many-body potential trained by force matching on the GPU, with
a force-matched pair table (VerletListTabulated) as the fallback.

Every simulation and force evaluation runs in the CUDA library; numpy only moves frames,
builds histograms and solves the small least-squares problem of the pair-table fit.
"""
import ctypes
import math
import os

import numpy as np

from . import _abi
from ._abi import call, dptr, i32ptr, i64ptr
from ._lib import load_library
from .tools import topology

RC_WCA = 2.0 ** (1.0 / 6.0)
SKIN = 0.3


class Handle:
    """A system of the CUDA library driven through the C ABI."""

    def __init__(self, box, skin, cutoff, precision=_abi.PREC_MIXED, seed=1, lib=None):
        self.lib = lib or load_library()
        self.box = np.asarray(box, np.float64)
        cg = np.array([max(3, int(b / (cutoff + skin))) for b in self.box], np.int32)
        self.h = ctypes.c_void_p()
        call(self.lib, "espp_system_create", dptr(self.box), skin, i32ptr(cg), precision, seed,
             ctypes.byref(self.h))

    def close(self):
        if self.h:
            self.lib.espp_system_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, ids, pos, mass=None):
        ids = np.ascontiguousarray(ids, np.int64)
        m = None if mass is None else np.ascontiguousarray(np.broadcast_to(mass, ids.shape),
                                                           np.float64)
        call(self.lib, "espp_add_particles", self.h, len(ids), i64ptr(ids), None, dptr(m),
             dptr(np.ascontiguousarray(pos, np.float64).reshape(-1)), None)
        call(self.lib, "espp_decompose", self.h)

    def set_pos(self, ids, pos):
        call(self.lib, "espp_set_particles", self.h, len(ids), i64ptr(ids),
             dptr(np.ascontiguousarray(pos, np.float64).reshape(-1)), None)

    def state(self, ids):
        n = len(ids)
        pos, vel, frc = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
        img = np.zeros((n, 3), np.int32)
        call(self.lib, "espp_get_particles", self.h, n, i64ptr(ids), dptr(pos), dptr(vel),
             dptr(frc), i32ptr(img))
        return pos, vel, frc, img

    def run(self, n):
        call(self.lib, "espp_run", self.h, int(n))

    def energy(self, which):
        e = ctypes.c_double()
        call(self.lib, "espp_energy", self.h, which, ctypes.byref(e))
        return e.value

    def rdf(self, nbins):
        g = np.zeros(nbins)
        call(self.lib, "espp_rdf", self.h, nbins, dptr(g))
        return g


# ---- fine-grained melt ------------------------------------------------------------
def fg_melt(nchains, nbeads, seed=3, precision=_abi.PREC_MIXED, thermostat=True, lib=None):
    """Kremer-Grest melt at density 0.85: WCA + FENE(30, 1.5), dt 0.01, Langevin gamma 0.5
    T 1 (thermostat=True).  The pair force starts capped (caprad 0.9); fg_uncap() ends
    the warm-up.  Returns (handle, ids, bonds, L)."""
    pos, bonds, L = topology.polymer_melt(nchains, nbeads, 0.85, seed=seed)
    h = Handle([L, L, L], SKIN, RC_WCA, precision, seed=seed + 100, lib=lib)
    ids = np.arange(1, len(pos) + 1, dtype=np.int64)
    h.add(ids, pos)
    fg_potentials(h, bonds, caprad=0.9)
    call(h.lib, "espp_integrator_set", h.h, 0.01)
    if thermostat:
        call(h.lib, "espp_langevin_set", h.h, 1, 0.5, 1.0, 0, None)
    return h, ids, bonds, L


def fg_potentials(h, bonds, caprad=0.0):
    call(h.lib, "espp_vl_create", h.h, RC_WCA, 0, None)
    fg_lj(h, caprad)
    b = np.ascontiguousarray(bonds, np.int64).reshape(-1)
    call(h.lib, "espp_bonds_add", h.h, len(b) // 2, i64ptr(b))
    call(h.lib, "espp_fene_set", h.h, 30.0, 0.0, 1.5, math.inf, 0.0)


def fg_lj(h, caprad):
    shift = 4.0 * (RC_WCA ** -12 - RC_WCA ** -6)
    call(h.lib, "espp_lj_set", h.h, 0, 0, 1.0, 1.0, RC_WCA, shift, caprad)


def map_frame(pos_unwrapped, forces, nper):
    """Centres of mass of consecutive groups of nper beads (equal masses) and the summed
    forces of each group."""
    n = len(pos_unwrapped) // nper
    com = pos_unwrapped[: n * nper].reshape(n, nper, 3).mean(axis=1)
    f = forces[: n * nper].reshape(n, nper, 3).sum(axis=1)
    return com, f


def fg_frames(nchains, nbeads, nframes, interval, warm_capped=1000, warm=4000, nper=4, seed=3,
              window=1, lib=None, log=None):
    """Runs the fine-grained melt and returns mapped frames: CG positions (unwrapped,
    (F, M, 3)), mapped conservative forces (F, M, 3), the box length, and the CG bond list.
    window = 1: the forces of each frame's configuration, from a second copy of the melt
    without thermostat.  window > 1: the thermostat pauses for `window` steps, the mapped
    conservative forces are averaged over them on the device (espp_force_acc), and the
    positions are those of the middle step; averaging removes most of the fast bond
    vibration of the mapped force."""
    h, ids, bonds, L = fg_melt(nchains, nbeads, seed=seed, lib=lib)
    ref = None
    if window <= 1:
        ref = Handle([L, L, L], SKIN, RC_WCA, _abi.PREC_FP64, seed=seed, lib=h.lib)
        ref.add(ids, h.state(ids)[0])
        fg_potentials(ref, bonds)
    h.run(warm_capped)
    fg_lj(h, 0.0)
    h.run(warm)
    if log:
        log("fine-grained melt warmed up (%d + %d steps)" % (warm_capped, warm))
    m = len(ids) // nper
    pos = np.zeros((nframes, m, 3))
    frc = np.zeros((nframes, m, 3))
    for f in range(nframes):
        h.run(interval)
        if ref is not None:
            p, _, _, img = h.state(ids)
            ref.set_pos(ids, p)
            ref.run(0)
            fc = ref.state(ids)[2]
        else:
            call(h.lib, "espp_langevin_set", h.h, 0, 0.5, 1.0, 0, None)
            call(h.lib, "espp_force_acc", h.h, 0, 0, None, None)
            for w in range(window):
                h.run(1)
                call(h.lib, "espp_force_acc", h.h, 1, 0, None, None)
                if w == window // 2:
                    p, _, _, img = h.state(ids)
            fc = np.zeros((len(ids), 3))
            call(h.lib, "espp_force_acc", h.h, 2, len(ids), i64ptr(ids), dptr(fc))
            fc /= window
            call(h.lib, "espp_langevin_set", h.h, 1, 0.5, 1.0, 0, None)
        pos[f], frc[f] = map_frame(p + img * L, fc, nper)
    h.close()
    if ref is not None:
        ref.close()
    site = np.arange(1, m + 1, dtype=np.int64).reshape(nchains, nbeads // nper)
    cg_bonds = np.stack([site[:, :-1].reshape(-1), site[:, 1:].reshape(-1)], 1)
    return pos, frc, L, cg_bonds


# ---- coarse-grained interactions --------------------------------------------------
def wrap(pos, L):
    return pos - L * np.floor(pos / L)


def bond_lengths(pos_unwrapped, cg_bonds):
    d = pos_unwrapped[:, cg_bonds[:, 1] - 1] - pos_unwrapped[:, cg_bonds[:, 0] - 1]
    return np.sqrt(np.sum(d * d, axis=-1)).ravel()


def write_table(path, r, e, f):
    with open(path, "w") as out:
        for a, b, c in zip(r, e, f):
            out.write("%15.8g %15.8g %15.8g\n" % (a, b, c))


def boltzmann_bond_table(lengths, T=1.0, n=400, rmin=0.05, rmax=8.0, path=None):
    """Bond potential U(r) = -T ln(P(r) / r^2) from the bond-length histogram, harmonic
    continuation outside the sampled range, force -dU/dr; returns (r, E, F)."""
    lo, hi = np.percentile(lengths, [0.2, 99.8])
    nb = 60
    hist, edges = np.histogram(lengths, bins=nb, range=(lo, hi), density=True)
    rc = 0.5 * (edges[1:] + edges[:-1])
    ok = hist > 0
    u = -T * np.log(hist[ok] / rc[ok] ** 2)
    # quadratic fit of U(r) carries the potential smoothly outside the sampled range
    a2, a1, a0 = np.polyfit(rc[ok], u, 2)
    a2 = max(a2, 1.0)
    r = np.linspace(rmin, rmax, n)
    uq = a2 * r * r + a1 * r + a0
    ui = np.interp(r, rc[ok], u)
    inside = (r >= rc[ok][0]) & (r <= rc[ok][-1])
    w = np.exp(-((r - np.clip(r, rc[ok][0], rc[ok][-1])) / 0.05) ** 2)
    U = np.where(inside, ui, w * np.interp(r, rc[ok], u) + (1 - w) * uq)
    U = np.convolve(np.pad(U, 3, mode="edge"), np.ones(7) / 7, mode="valid")
    U -= U.min()
    F = -np.gradient(U, r)
    if path:
        write_table(path, r, U, F)
    return r, U, F


def angle_triples(cg_bonds):
    """Triples (a, b, c) of consecutive sites of a chain: bonds (a, b) and (b, c)."""
    bs = {(int(a), int(b)) for a, b in np.asarray(cg_bonds).reshape(-1, 2)}
    return np.array([(a, b, b + 1) for a, b in sorted(bs) if b == a + 1 and (b, b + 1) in bs],
                    np.int64).reshape(-1, 3)


def angles_of(pos_unwrapped, triples):
    """Bending angles theta (radians) of the triples in every frame (frames, N, 3)."""
    p = np.asarray(pos_unwrapped)
    t = np.asarray(triples) - 1
    d12 = p[:, t[:, 0]] - p[:, t[:, 1]]
    d32 = p[:, t[:, 2]] - p[:, t[:, 1]]
    c = np.sum(d12 * d32, -1) / np.sqrt(np.sum(d12 * d12, -1) * np.sum(d32 * d32, -1))
    return np.arccos(np.clip(c, -1.0, 1.0)).reshape(-1)


def boltzmann_angle_table(thetas, T=1.0, n=721, nbins=90, stiff=20.0, path=None):
    """Angle potential U(theta) = -T ln(P(theta) / sin(theta)) from the angle histogram,
    smoothed; below the sampled range a stiff quadratic wall, and near theta = pi the
    quadratic through the last sampled bins, so that U is flat at pi and the tabulated
    angular force f / sin(theta) stays finite there.  Returns (theta, E, f = -dE/dtheta)."""
    hist, edges = np.histogram(thetas, bins=nbins, range=(0.0, math.pi), density=True)
    tc = 0.5 * (edges[1:] + edges[:-1])
    ok = hist > 0.002 * hist.max()
    u = np.full(nbins, np.nan)
    u[ok] = -T * np.log(hist[ok] / np.sin(tc[ok]))
    first = int(np.argmax(ok))
    th = np.linspace(0.0, math.pi, n)
    U = np.interp(th, tc[ok], u[ok])
    lo = tc[first]
    U = np.where(th < lo, U[np.searchsorted(th, lo)] + stiff * (lo - th) ** 2, U)
    # flat at pi: even quadratic in (pi - theta) fitted to the last sampled bins
    tail = ok & (tc > math.pi - 0.6)
    if np.count_nonzero(tail) >= 3:
        x = (math.pi - tc[tail]) ** 2
        c1, c0 = np.polyfit(x, u[tail], 1)
        near = th > math.pi - 0.3
        w = np.clip((th - (math.pi - 0.3)) / 0.3, 0.0, 1.0)
        U = np.where(near, (1 - w) * U + w * (c0 + c1 * (math.pi - th) ** 2), U)
    U = np.convolve(np.pad(U, 4, mode="edge"), np.ones(9) / 9, mode="valid")
    U -= U.min()
    F = -np.gradient(U, th)
    F[-1] = 0.0
    if path:
        write_table(path, th, U, F)
    return th, U, F


def pair_fm_table(frames_pos, frames_f, L, rc=3.0, nknots=50, wall=100.0, path=None,
                  exclude=None):
    """Force-matched radial pair force f(r): hat functions on nknots points from the
    closest sampled separation to rc, fitted by regularised linear least squares to the
    target forces; below the sampled range a repulsive wall (slope `wall`).  Pairs of
    `exclude` (site id pairs, e.g. the bonds) take no part.  The fallback of the learned
    potential, and its prior.  Returns the table (r, E, F) with E = integral of f from r
    to rc."""
    from scipy.spatial import cKDTree
    ex = None
    if exclude is not None and len(exclude):
        e = np.sort(np.asarray(exclude, np.int64).reshape(-1, 2) - 1, axis=1)
        ex = set(map(tuple, e.tolist()))
    pair_sets = []
    for pos in frames_pos:
        p = wrap(pos, L)
        pairs = cKDTree(p, boxsize=L).query_pairs(rc, output_type="ndarray")
        if ex is not None:
            keep = np.array([(int(a), int(b)) not in ex for a, b in pairs], bool)
            pairs = pairs[keep]
        d = p[pairs[:, 0]] - p[pairs[:, 1]]
        d -= L * np.round(d / L)
        pair_sets.append((pairs, d, np.sqrt(np.sum(d * d, 1))))
    rlo = float(min(q[2].min() for q in pair_sets))
    knots = np.linspace(rlo, rc, nknots)
    h = knots[1] - knots[0]
    M = np.zeros((nknots, nknots))
    b = np.zeros(nknots)
    for (pairs, d, r), f, pos in zip(pair_sets, frames_f, frames_pos):
        rh = d / r[:, None]
        t = np.clip((r - rlo) / h, 0, nknots - 1 - 1e-9)
        k0 = t.astype(int)
        w1 = t - k0
        A = np.zeros((len(pos), 3, nknots))
        for kk, ww in ((k0, 1 - w1), (k0 + 1, w1)):
            contrib = rh * ww[:, None]
            np.add.at(A, (pairs[:, 0], slice(None), kk), contrib)
            np.add.at(A, (pairs[:, 1], slice(None), kk), -contrib)
        A2 = A.reshape(-1, nknots)
        M += A2.T @ A2
        b += A2.T @ f.reshape(-1)
    lam = 1e-6 * np.trace(M) / nknots
    D = np.diff(np.eye(nknots), 2, axis=0)
    coef = np.linalg.solve(M + lam * np.eye(nknots) + 10 * lam * D.T @ D, b)
    r = np.linspace(0.05, rc, 400)
    fr = np.interp(r, knots, coef)
    below = r < rlo
    fr[below] = coef[0] + (rlo - r[below]) * wall
    E = np.zeros_like(r)
    E[:-1] = np.cumsum(((fr[:-1] + fr[1:]) * 0.5 * np.diff(r))[::-1])[::-1]
    if path:
        write_table(path, r, E, fr)
    return r, E, fr


class CGSystem(Handle):
    """CG sites (mass = beads per site) with the bond table and, optionally, the learned
    potential or the pair-table fallback on a Verlet list of cutoff rc."""

    def __init__(self, pos, L, cg_bonds, bond_tab, mass=4.0, rc=3.0, precision=_abi.PREC_MIXED,
                 seed=5, lib=None, exclude=None):
        Handle.__init__(self, [L, L, L], SKIN, rc, precision, seed=seed, lib=lib)
        self.L = L
        self.ids = np.arange(1, len(pos) + 1, dtype=np.int64)
        self.add(self.ids, wrap(pos, L), mass=mass)
        if exclude is not None and len(exclude):
            ex = np.ascontiguousarray(exclude, np.int64).reshape(-1)
            call(self.lib, "espp_vl_create", self.h, rc, len(ex) // 2, i64ptr(ex))
        else:
            call(self.lib, "espp_vl_create", self.h, rc, 0, None)
        b = np.ascontiguousarray(cg_bonds, np.int64).reshape(-1)
        call(self.lib, "espp_bonds_add", self.h, len(b) // 2, i64ptr(b))
        self.set_bond_table(bond_tab)
        self.mlp = None

    def set_bond_table(self, tab):
        # linear interpolation: beyond the table the force continues linearly
        r, e, f = (np.ascontiguousarray(a, np.float64) for a in tab)
        call(self.lib, "espp_tab_bond_set", self.h, 1, len(r), dptr(r), dptr(e), dptr(f),
             math.inf, 0.0)

    def set_angle_table(self, triples, tab):
        """FixedTripleListTabulatedAngular on the triples (linear interpolation)."""
        t = np.ascontiguousarray(triples, np.int64).reshape(-1)
        call(self.lib, "espp_triples_add", self.h, len(t) // 3, i64ptr(t))
        th, e, f = (np.ascontiguousarray(a, np.float64) for a in tab)
        call(self.lib, "espp_tab_angle_set", self.h, 1, len(th), dptr(th), dptr(e), dptr(f))

    def set_pair_table(self, tab, rc=3.0):
        r, e, f = (np.ascontiguousarray(a, np.float64) for a in tab)
        call(self.lib, "espp_tab_pair_set", self.h, 0, 0, 1, len(r), dptr(r), dptr(e), dptr(f),
             rc, 0.0)

    def attach(self, model):
        self.mlp = model
        call(self.lib, "espp_mlp_attach", self.h, model.m if model else None)

    def thermostat(self, on, gamma=0.5, T=1.0):
        self.langevin = (gamma, T) if on else None
        call(self.lib, "espp_langevin_set", self.h, 1 if on else 0, gamma, T, 0, None)

    def forces_at(self, pos):
        """Conservative forces at the configuration pos (the thermostat is paused)."""
        lv = getattr(self, "langevin", None)
        if lv:
            call(self.lib, "espp_langevin_set", self.h, 0, lv[0], lv[1], 0, None)
        self.set_pos(self.ids, wrap(pos, self.L))
        self.run(0)
        if lv:
            call(self.lib, "espp_langevin_set", self.h, 1, lv[0], lv[1], 0, None)
        return self.state(self.ids)[2]


class MLPModel:
    """A learned potential of the library (weights on the device)."""

    def __init__(self, rc=3.0, r0=0.5, seed=1, lib=None):
        self.lib = lib or load_library()
        self.m = ctypes.c_void_p()
        call(self.lib, "espp_mlp_create", rc, r0, ctypes.byref(self.m))
        n = ctypes.c_int64()
        call(self.lib, "espp_mlp_num_params", ctypes.byref(n))
        self.nparams = n.value
        rng = np.random.Generator(np.random.PCG64(seed))
        K, H = 16, 64
        # small output layer: the untrained model adds little to its prior
        theta = np.concatenate([rng.normal(0, 1 / math.sqrt(K), H * K), np.zeros(H),
                                rng.normal(0, 1 / math.sqrt(H), H * H), np.zeros(H),
                                rng.normal(0, 0.01 / math.sqrt(H), H), [0.0]])
        self.set_params(theta)

    def set_params(self, theta):
        call(self.lib, "espp_mlp_set_params", self.m, self.nparams,
             dptr(np.ascontiguousarray(theta, np.float64)))

    def params(self):
        t = np.zeros(self.nparams)
        call(self.lib, "espp_mlp_get_params", self.m, self.nparams, dptr(t))
        return t

    def set_norm(self, shift, scale):
        call(self.lib, "espp_mlp_set_norm", self.m, dptr(np.ascontiguousarray(shift, np.float64)),
             dptr(np.ascontiguousarray(scale, np.float64)))

    def close(self):
        if self.m:
            self.lib.espp_mlp_destroy(self.m)
            self.m = ctypes.c_void_p()


def descriptor_norm(cg, frames_pos, nframes=4):
    """Mean and inverse standard deviation of the descriptors over a few frames."""
    G = []
    for pos in frames_pos[:nframes]:
        cg.set_pos(cg.ids, wrap(pos, cg.L))
        call(cg.lib, "espp_decompose", cg.h)
        g = np.zeros((len(cg.ids), 16))
        call(cg.lib, "espp_mlp_descriptors", cg.h, len(cg.ids), i64ptr(cg.ids), dptr(g))
        G.append(g)
    G = np.concatenate(G)
    # components that barely vary (basis functions below the closest approach) are not
    # amplified: the variance floor is 1 % of the largest component's
    sd = G.std(0)
    return G.mean(0), 1.0 / np.sqrt(sd * sd + (0.1 * sd.max()) ** 2)


def train_mlp(cg, model, frames_pos, frames_target, epochs=10, batch=4, lr=2e-3, seed=0,
              log=None):
    """Force matching on the GPU: for every frame the library evaluates the loss and its
    gradient (espp_mlp_fm_grad); Adam steps every `batch` frames.  Returns the mean loss of
    each epoch."""
    rng = np.random.Generator(np.random.PCG64(seed))
    hist = []
    nf = len(frames_pos)
    for ep in range(epochs):
        order = rng.permutation(nf)
        tot = 0.0
        for k, f in enumerate(order):
            cg.set_pos(cg.ids, wrap(frames_pos[f], cg.L))
            call(cg.lib, "espp_decompose", cg.h)
            loss = ctypes.c_double()
            call(cg.lib, "espp_mlp_fm_grad", cg.h, len(cg.ids), i64ptr(cg.ids),
                 dptr(np.ascontiguousarray(frames_target[f], np.float64).reshape(-1)),
                 ctypes.byref(loss), None)
            tot += loss.value
            if (k + 1) % batch == 0 or k + 1 == nf:
                step_lr = lr * 0.5 * (1 + math.cos(math.pi * (ep + k / nf) / epochs))
                call(cg.lib, "espp_mlp_adam_step", model.m, step_lr, 0.9, 0.999, 1e-8,
                     1.0 / batch)
        hist.append(tot / nf)
        if log:
            log("epoch %d: force-matching loss %.4f" % (ep, hist[-1]))
    return hist


def fm_error(cg, frames_pos, frames_target, frames_sub=None):
    """Relative force-matching error sqrt(sum |F - F_target|^2 / sum |F_target|^2) over
    the given frames, F the system's force minus frames_sub (a known part, e.g. the bond
    forces) when given."""
    num = den = 0.0
    for k, (pos, tgt) in enumerate(zip(frames_pos, frames_target)):
        f = cg.forces_at(pos)
        if frames_sub is not None:
            f = f - frames_sub[k]
        num += float(np.sum((f - tgt) ** 2))
        den += float(np.sum(tgt ** 2))
    return math.sqrt(num / den)


def chain_com_msd(pos_series, sites_per_chain):
    """Mean squared displacement of chain centres of mass between the first and each
    later configuration of a series of unwrapped site positions (T, M, 3)."""
    T, M, _ = pos_series.shape
    com = pos_series.reshape(T, M // sites_per_chain, sites_per_chain, 3).mean(axis=2)
    d = com - com[0]
    return np.mean(np.sum(d * d, axis=-1), axis=1)


def rdf_of_frames(cg, frames_pos, nbins):
    g = np.zeros(nbins)
    for pos in frames_pos:
        cg.set_pos(cg.ids, wrap(pos, cg.L))
        g += cg.rdf(nbins)
    return g / len(frames_pos)


def ibi_refine(cgsys, tab, g_target, nbins, iters=10, steps=3000, every=250, alpha=0.8,
               rc=3.0, T=1.0, log=None, bonded=None):
    """Iterative Boltzmann inversion of a pair table against a target RDF: each iteration
    runs the CG system (bonds + this pair table, thermostatted) on the GPU, samples the
    RDF, and updates U(r) += alpha T ln(g(r) / g_target(r)) (step at most alpha T, bins
    where either RDF is sampled, tapered to zero at rc); F = -dU/dr.  An iteration whose RDF error
    is larger than the best so far goes back to the best tables and halves alpha, and the
    best tables are the ones returned.
    bonded = (bonds, bond table, target bond lengths): the bond table is refined in the
    same way against the bond-length distribution of the target (U_b += alpha T
    ln(P(r) / P_target(r)) over the sampled range).
    Returns the refined pair table, the RDF L2 error per iteration, and the last sampled
    RDF of the best tables."""
    r_t, E_t, F_t = (np.array(a, np.float64) for a in tab)
    dr = cgsys.L / 2 / nbins
    rb = (np.arange(nbins) + 0.5) * dr
    hist = []
    if bonded is not None:
        bonds, btab, blen = bonded
        rbt, Ebt, _ = (np.array(a, np.float64) for a in btab)
        lo, hi = np.percentile(blen, [0.5, 99.5])
        bedges = np.linspace(lo, hi, 41)
        pb_target, _ = np.histogram(blen, bins=bedges, density=True)
        bc = 0.5 * (bedges[1:] + bedges[:-1])
        bidx = np.asarray(bonds, np.int64).reshape(-1, 2) - 1
    best = (np.inf, E_t.copy(), None, None if bonded is None else Ebt.copy(), None)
    for it in range(iters):
        cgsys.set_pair_table((r_t, E_t, F_t), rc)
        if bonded is not None:
            cgsys.set_bond_table((rbt, Ebt, -np.gradient(Ebt, rbt)))
        cgsys.run(1000)
        g = np.zeros(nbins)
        lens = []
        ns = 0
        for _ in range(steps // every):
            cgsys.run(every)
            g += cgsys.rdf(nbins)
            if bonded is not None:
                p = cgsys.state(cgsys.ids)[0]
                d = p[bidx[:, 0]] - p[bidx[:, 1]]
                d -= cgsys.L * np.round(d / cgsys.L)
                lens.append(np.sqrt(np.sum(d * d, 1)))
            ns += 1
        g /= ns
        pb = None
        if bonded is not None:
            pb, _ = np.histogram(np.concatenate(lens), bins=bedges, density=True)
        sel = rb < 2 * rc
        hist.append(float(np.sqrt(np.mean((g[sel] - g_target[sel]) ** 2))))
        if log:
            log("IBI iteration %d: RDF L2 %.4f (alpha %.3f)" % (it, hist[-1], alpha))
        if hist[-1] < best[0]:
            best = (hist[-1], E_t.copy(), g.copy(), None if bonded is None else Ebt.copy(), pb)
        else:
            # overshoot: step again from the best tables with half the step
            alpha *= 0.5
            E_t = best[1].copy()
            g = best[2]
            if bonded is not None:
                Ebt = best[3].copy()
                pb = best[4]
        # bins where either RDF is sampled (the core too, where the CG sites come closer
        # than the mapped ones); steps of at most alpha T per iteration
        ok = (rb < rc) & ((g > 0.002) | (g_target > 0.002))
        du = np.zeros(nbins)
        du[ok] = alpha * T * np.clip(
            np.log(np.maximum(g[ok], 1e-4) / np.maximum(g_target[ok], 1e-4)), -1.0, 1.0)
        du = np.convolve(du, np.ones(3) / 3, mode="same")
        first = np.argmax(ok)
        du[:first] = du[first]
        du *= np.clip(1.0 - (rb / rc) ** 4, 0.0, 1.0)
        E_t = E_t + np.interp(r_t, rb, du)
        F_t = -np.gradient(E_t, r_t)
        if bonded is not None:
            okb = (pb > 0.01 * pb_target.max()) & (pb_target > 0.01 * pb_target.max())
            dub = np.zeros_like(bc)
            dub[okb] = alpha * T * np.clip(np.log(pb[okb] / pb_target[okb]), -1.0, 1.0)
            dub = np.convolve(dub, np.ones(3) / 3, mode="same")
            # over the sampled range; outside it the end values (a constant shift keeps the
            # continuation's force)
            if okb.any():
                Ebt = Ebt + np.interp(rbt, bc[okb], dub[okb])
    E_t = best[1]
    F_t = -np.gradient(E_t, r_t)
    cgsys.set_pair_table((r_t, E_t, F_t), rc)
    if bonded is not None:
        cgsys.set_bond_table((rbt, best[3], -np.gradient(best[3], rbt)))
    return (r_t, E_t, F_t), hist, best[2]
