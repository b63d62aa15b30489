"""Spatial domain decomposition of one periodic box over several GPUs.

The reference decomposes space over MPI ranks: each rank owns the particles of its block
of cells, keeps ghost copies of the neighbouring ranks' boundary cells (refreshed every
step, src/storage/DomainDecomposition.cpp:1243-1391) and moves particles between ranks
when it re-sorts (decomposeRealParticles, :1031-1158); a re-sort is decided by the global
maximum displacement (VelocityVerlet.cpp:63-169).  Here the box is cut into slabs of
whole cells along z, one slab per domain and one system of the C ABI per domain (one
domain per GPU).  A domain's system holds the particles it owns and halo copies of the
particles in the h cell layers (h = halfCellInt) on either side of its slab; the halo
copies are partners only (the library does not integrate, thermostat or count them).

Every step the owners send the new positions of the particles other domains hold as halo
copies; at a re-sort the domains send each of their particles to its new owner and, as a
halo copy, to every domain whose halo layer holds it.  The communicator is either
``LocalComm`` (all domains in this process, e.g. several domains on one device) or
``TorchComm`` (one process per rank over ``torch.distributed``: NCCL between GPUs, gloo
on CPU).  Cell membership is computed on the host with the library's own fold and cell
map (the same rounded operations), so a particle's owner always holds it in one of the
owner's cells.

Supported on decomposed systems: Lennard-Jones (capped too), tabulated pairs and bonds,
FENE bonds, Verlet-list exclusions, Langevin (with exclusions), CapForce, energies,
virials, kinetic sums, pair sets.  Angles, the learned potential and the RDF need the
whole system and are refused.
"""
import ctypes
import math

import numpy as np

from . import _abi
from ._abi import call, dptr, i32ptr, i64ptr, u8ptr
from ._lib import load_library


class LocalComm:
    """Every domain lives in this process."""

    rank = 0
    world = 1

    def allgather(self, obj):
        return [obj]


class TorchComm:
    """One process per rank; objects are exchanged with torch.distributed's
    all_gather_object (the default group unless one is given)."""

    def __init__(self, dist=None, group=None):
        if dist is None:
            import torch.distributed as dist
        self._dist = dist
        self._group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def allgather(self, obj):
        out = [None] * self.world
        self._dist.all_gather_object(out, obj, group=self._group)
        return out


def fold_cells(x, L, nc):
    """The library's fold and cell map along one axis (k_fold_bin / the oracle's
    foldCoordinate + mapChecked): folded coordinate, image shift and cell index, with
    the same rounded operations."""
    x = np.asarray(x, np.float64)
    inv_l = 1.0 / L
    tmp = np.floor(x * inv_l).astype(np.int64)
    xf = x - tmp.astype(np.float64) * L
    inv_cell = 1.0 / ((L - 0.0) / float(nc))
    t = xf * inv_cell
    c = np.clip(np.trunc(t), 0, nc - 1).astype(np.int64)
    return xf, tmp, c


def slab_bounds(nz, ndomains):
    """Cells [z0, z1) of each domain's slab along z."""
    return [(d * nz // ndomains, (d + 1) * nz // ndomains) for d in range(ndomains)]


class _Failed:
    """An error of one rank, carried to all ranks by the next gather."""

    def __init__(self, msg):
        self.msg = msg


def _cat(parts, k, shape, dtype):
    return np.concatenate([p[k] for p in parts]) if parts else np.zeros(shape, dtype)


class SpatialDecomposition:
    """A periodic box of cell_grid cells cut into `ndomains` slabs along z (the reference's
    nodeGrid (1, 1, ndomains)).  This process drives the domains comm.rank * k ..
    (comm.rank + 1) * k - 1, k = ndomains / comm.world.  The calls mirror the C ABI of one
    system; observables are summed over all domains and returned on every rank."""

    def __init__(self, box, skin, cell_grid, ndomains, precision=_abi.PREC_FP64, seed=12345,
                 comm=None, lib=None, half_cell_int=1, exchange="host"):
        """exchange: how the per-step halo positions travel. "host": through host arrays
        (espp_get_particles / espp_dd_set_halo_positions, gathered with the communicator);
        "direct": in buffers of the library's memory space (device memory for the CUDA
        library), copied between domains of this process and sent between ranks with
        torch.distributed point-to-point operations (NCCL between GPUs, gloo on CPU)."""
        self.comm = comm or LocalComm()
        self.lib = lib or load_library()
        if exchange not in ("host", "direct"):
            raise ValueError("exchange must be 'host' or 'direct'")
        self.exchange = exchange
        self.box = np.asarray(box, np.float64).copy()
        self.skin = float(skin)
        self.cg = np.asarray(cell_grid, np.int32).copy()
        self.h = int(half_cell_int)
        self.D = int(ndomains)
        if self.D < 1 or self.D % self.comm.world:
            raise ValueError("ndomains must be a positive multiple of the number of ranks")
        if self.D > int(self.cg[2]):
            raise ValueError("more domains than cells along z")
        per = self.D // self.comm.world
        self.local = list(range(self.comm.rank * per, (self.comm.rank + 1) * per))
        nz = int(self.cg[2])
        self.bounds = slab_bounds(nz, self.D)
        self.slab_of = np.empty(nz, np.int64)
        for d, (z0, z1) in enumerate(self.bounds):
            self.slab_of[z0:z1] = d
        # halo_of[e][cz]: cell layer cz lies within h cells of domain e's slab (and is not
        # e's own); one domain has no halo (the library's periodic wrap covers it)
        self.halo_of = np.zeros((self.D, nz), bool)
        if self.D > 1:
            for e, (z0, z1) in enumerate(self.bounds):
                for k in range(1, self.h + 1):
                    self.halo_of[e, (z0 - k) % nz] = True
                    self.halo_of[e, (z1 - 1 + k) % nz] = True
                self.halo_of[e, z0:z1] = False
        self.handles = {}
        for d in self.local:
            hd = ctypes.c_void_p()
            call(self.lib, "espp_system_create", dptr(self.box), self.skin, i32ptr(self.cg),
                 int(precision), int(seed), ctypes.byref(hd))
            if self.h != 1:
                call(self.lib, "espp_set_half_cell_int", hd, self.h)
            self.handles[d] = hd
        self.owned = {d: np.zeros(0, np.int64) for d in self.local}
        # halo copies each domain holds and the domain owning each of them
        self.halo = {d: (np.zeros(0, np.int64), np.zeros(0, np.int64)) for d in self.local}
        self.export = {d: {} for d in self.local}
        self.maxDist = 0.0
        self.resorts = 0
        self.last_resorts = 0  # re-sorts of the last run
        self._ids = np.zeros(0, np.int64)  # sorted ids and their types and masses
        self._type = np.zeros(0, np.int32)
        self._mass = np.zeros(0, np.float64)
        self._pending = None
        self._bonds = np.zeros((0, 2), np.int64)
        self._per = per
        self._xids = {}  # direct exchange: id arrays in the library's memory space
        self._hids = {}

    # ---- set-up -------------------------------------------------------------------
    def add_particles(self, ids, pos, vel=None, types=None, mass=None):
        """Storage.addParticles: every rank passes the whole set; decompose() hands each
        domain its particles."""
        ids = np.asarray(ids, np.int64)
        n = len(ids)
        pos = np.array(pos, np.float64).reshape(n, 3)
        vel = np.zeros((n, 3)) if vel is None else np.array(vel, np.float64).reshape(n, 3)
        types = np.zeros(n, np.int32) if types is None else np.asarray(types, np.int32)
        mass = np.ones(n) if mass is None else np.asarray(mass, np.float64)
        if len(np.unique(ids)) != n or np.isin(ids, self._ids).any():
            raise RuntimeError("duplicate particle id")
        # Storage::addParticle folds the position (the images start from the fold)
        img = np.zeros((n, 3), np.int32)
        for k in range(3):
            xf, tmp, _ = fold_cells(pos[:, k], self.box[k], int(self.cg[k]))
            pos[:, k] = xf
            img[:, k] = tmp
        allids = np.concatenate([self._ids, ids])
        order = np.argsort(allids, kind="stable")
        self._ids = allids[order]
        self._type = np.concatenate([self._type, types])[order]
        self._mass = np.concatenate([self._mass, mass])[order]
        rows = (ids, pos, vel, img)
        if self._pending is None:
            self._pending = rows
        else:
            self._pending = tuple(np.concatenate([a, b]) for a, b in zip(self._pending, rows))

    def decompose(self):
        """Storage.decompose: the particles added so far (and those already held) are
        distributed to their owners, with halo copies."""
        held = self._guarded(self._collect_owned)
        parts = self.comm.allgather(held if isinstance(held, _Failed) else self._bucket_all(held))
        self._raise_failed(parts)
        if self._pending is not None:
            # every rank passed the whole set of new particles: each buckets it itself
            parts.append(self._bucket_all(self._pending))
            self._pending = None
        self._load(parts)
        self._each("espp_decompose")
        self.maxDist = 0.0

    def _each(self, name, *args):
        for d in self.local:
            call(self.lib, name, self.handles[d], *args)

    def vl_create(self, cutoff, excl_pairs=None):
        ex = (None if excl_pairs is None
              else np.ascontiguousarray(excl_pairs, np.int64).reshape(-1))
        self._each("espp_vl_create", float(cutoff), 0 if ex is None else len(ex) // 2,
                   i64ptr(ex))

    def lj_set(self, t1, t2, eps, sig, rc, shift, caprad=0.0):
        self._each("espp_lj_set", int(t1), int(t2), float(eps), float(sig), float(rc),
                   float(shift), float(caprad))

    def fene_set(self, K=30.0, r0=0.0, rmax=1.5, rc=math.inf, shift=0.0):
        self._each("espp_fene_set", float(K), float(r0), float(rmax), float(rc), float(shift))

    def tab_pair_set(self, t1, t2, itype, r, e, f, rc, shift=0.0):
        r, e, f = (np.ascontiguousarray(a, np.float64) for a in (r, e, f))
        self._each("espp_tab_pair_set", int(t1), int(t2), int(itype), len(r), dptr(r),
                   dptr(e), dptr(f), float(rc), float(shift))

    def tab_bond_set(self, itype, r, e, f, rc=math.inf, shift=0.0):
        r, e, f = (np.ascontiguousarray(a, np.float64) for a in (r, e, f))
        self._each("espp_tab_bond_set", int(itype), len(r), dptr(r), dptr(e), dptr(f),
                   float(rc), float(shift))

    def bonds_add(self, pairs):
        """FixedPairList.addBonds: each domain keeps the bonds of its owned particles."""
        b = np.sort(np.asarray(pairs, np.int64).reshape(-1, 2), axis=1)
        self._bonds = np.concatenate([self._bonds, b])
        for d in self.local:
            self._push_bonds(d)

    def integrator_set(self, dt):
        self._each("espp_integrator_set", float(dt))

    def langevin_set(self, enabled, gamma, temperature, excl=None):
        ex = None if excl is None else np.ascontiguousarray(excl, np.int64)
        self._each("espp_langevin_set", int(bool(enabled)), float(gamma), float(temperature),
                   0 if ex is None else len(ex), i64ptr(ex))

    def capforce_set(self, mode, cap):
        c = np.ascontiguousarray(np.broadcast_to(np.asarray(cap, np.float64), (3,)))
        self._each("espp_capforce_set", int(mode), dptr(c))

    # ---- the step loop ------------------------------------------------------------
    def run(self, nsteps):
        """VelocityVerlet.run(nsteps) over all domains: the start-of-run force, then per
        step the global re-sort decision, migration or halo refresh, force and
        integration."""
        nsteps = int(nsteps)
        self.last_resorts = 0
        m = self._global_max(self._guarded(
            lambda: [self._phase("espp_dd_run_begin", d, nsteps) for d in self.local]))
        for _ in range(nsteps):
            self.maxDist = self.maxDist + m
            resort = self.maxDist > 0.5 * self.skin
            pending = None
            if resort:
                self.maxDist = 0.0
                self.resorts += 1
                self.last_resorts += 1
                held = self._guarded(self._collect_owned)
                parts = self.comm.allgather(
                    held if isinstance(held, _Failed) else self._bucket_all(held))
                self._raise_failed(parts)
                self._load(parts)
            else:
                pending = self._refresh_halo()
            step = pending if isinstance(pending, _Failed) else self._guarded(
                lambda: [self._phase("espp_dd_step", d, int(resort)) for d in self.local])
            m = self._global_max(step)
        for d in self.local:
            call(self.lib, "espp_dd_run_end", self.handles[d])

    def _phase(self, name, d, arg):
        out = ctypes.c_double()
        call(self.lib, name, self.handles[d], arg, ctypes.byref(out))
        return out.value

    def _guarded(self, fn):
        """fn's result, or the error it raised as a _Failed value that the next gather
        turns into an error on every rank (esutil::Error, Error.cpp:52-64: the ranks'
        errors are collected and thrown together instead of leaving the others waiting)."""
        try:
            return fn()
        except Exception as e:  # noqa: BLE001 - reported to every rank below
            return _Failed("rank %d: %s" % (self.comm.rank, e))

    @staticmethod
    def _raise_failed(parts):
        errs = [p.msg for p in parts if isinstance(p, _Failed)]
        if errs:
            raise RuntimeError("; ".join(errs))

    def _global_max(self, values):
        parts = self.comm.allgather(values)
        self._raise_failed(parts)
        return max(max(v) if v else 0.0 for v in parts)

    # ---- migration and halo refresh ----------------------------------------------
    def _lookup(self, ids):
        k = np.searchsorted(self._ids, ids)
        return self._type[k], self._mass[k]

    def _collect_owned(self):
        """(ids, pos, vel, img) of the particles this process's domains own."""
        out = [np.zeros(0, np.int64), np.zeros((0, 3)), np.zeros((0, 3)),
               np.zeros((0, 3), np.int32)]
        for d in self.local:
            ids = self.owned[d]
            if len(ids) == 0:
                continue
            pos = np.zeros((len(ids), 3))
            vel = np.zeros((len(ids), 3))
            img = np.zeros((len(ids), 3), np.int32)
            call(self.lib, "espp_get_particles", self.handles[d], len(ids), i64ptr(ids),
                 dptr(pos), dptr(vel), None, i32ptr(img))
            for k, a in enumerate((ids, pos, vel, img)):
                out[k] = np.concatenate([out[k], a])
        return tuple(out)

    def _bucket_all(self, held):
        """{destination domain: (owned rows, halo rows, owners of the halo rows)} for the
        held particles; the owner is the slab of the particle's folded z cell."""
        ids, pos, vel, img = held
        _, _, cz = fold_cells(pos[:, 2], self.box[2], int(self.cg[2]))
        owner = self.slab_of[cz]
        out = {}
        for e in range(self.D):
            own = owner == e
            halo = self.halo_of[e, cz] & ~own
            if own.any() or halo.any():
                out[e] = ((ids[own], pos[own], vel[own], img[own]),
                          (ids[halo], pos[halo], vel[halo], img[halo]), owner[halo])
        return out

    def _load(self, gathered):
        """Replaces every local domain's particles with the rows sent to it."""
        failed = self._guarded(lambda: self._load_local(gathered))
        # who exports what: domain d sends to e the positions of the halo copies e holds
        # of d's particles (the receivers tell the owners); a load error travels along
        want = failed if isinstance(failed, _Failed) else {
            e: {int(o): self.halo[e][0][self.halo[e][1] == o]
                for o in np.unique(self.halo[e][1])} for e in self.local}
        gathered = self.comm.allgather(want)
        self._raise_failed(gathered)
        for d in self.local:
            self.export[d] = {e: ids for w in gathered for e, per in w.items()
                              for o, ids in per.items() if o == d}
        if self.exchange == "direct":
            self._xids = {d: {e: self._space(ids) for e, ids in sorted(self.export[d].items())}
                          for d in self.local}
            self._hids = {e: {o: self._space(w) for o, w in sorted(want[e].items())}
                          for e in self.local}

    def _load_local(self, gathered):
        for e in self.local:
            mine = [b[e] for b in gathered if e in b]
            own = [m[0] for m in mine]
            hal = [m[1] for m in mine]
            src = np.concatenate([m[2] for m in mine]) if mine else np.zeros(0, np.int64)
            ids_o = _cat(own, 0, 0, np.int64)
            ids_h = _cat(hal, 0, 0, np.int64)
            ids = np.concatenate([ids_o, ids_h])
            pos = np.concatenate([_cat(own, 1, (0, 3), float), _cat(hal, 1, (0, 3), float)])
            vel = np.concatenate([_cat(own, 2, (0, 3), float), _cat(hal, 2, (0, 3), float)])
            img = np.concatenate([_cat(own, 3, (0, 3), np.int32),
                                  _cat(hal, 3, (0, 3), np.int32)])
            halo = np.concatenate([np.zeros(len(ids_o), np.uint8),
                                   np.ones(len(ids_h), np.uint8)])
            ty, ms = self._lookup(ids)
            call(self.lib, "espp_dd_load", self.handles[e], len(ids), i64ptr(ids),
                 i32ptr(np.ascontiguousarray(ty, np.int32)),
                 dptr(np.ascontiguousarray(ms, np.float64)), dptr(np.ascontiguousarray(pos)),
                 dptr(np.ascontiguousarray(vel)), i32ptr(np.ascontiguousarray(img)),
                 u8ptr(halo))
            self.owned[e] = ids_o
            self.halo[e] = (ids_h, src)
            self._push_bonds(e)

    def _space(self, a):
        """A torch tensor with a's contents in the library's memory space."""
        import torch
        if not hasattr(self, "_device"):
            kind = ctypes.c_int32()
            call(self.lib, "espp_memory_space", ctypes.byref(kind))
            self._device = (torch.device("cuda", torch.cuda.current_device())
                            if kind.value == 1 else torch.device("cpu"))
        return torch.as_tensor(np.ascontiguousarray(a)).to(self._device)

    @staticmethod
    def _ptr(t, ctype):
        return ctypes.cast(t.data_ptr(), ctypes.POINTER(ctype))

    def _refresh_halo(self):
        """Every owner sends the current positions of its particles that other domains
        hold as halo copies (the reference's per-step ghost update).  Returns None, or a _Failed that the caller passes on to the next gather."""
        if self.exchange == "direct":
            return self._refresh_halo_direct()
        parts = self.comm.allgather(self._guarded(self._halo_rows))
        self._raise_failed(parts)
        return self._guarded(lambda: self._write_halo_rows(parts))

    def _halo_rows(self):
        out = {}
        for d in self.local:
            ex = self.export[d]
            if not ex:
                continue
            allids = np.concatenate(list(ex.values()))
            pos = np.zeros((len(allids), 3))
            call(self.lib, "espp_get_particles", self.handles[d], len(allids), i64ptr(allids),
                 dptr(pos), None, None, None)
            o = 0
            for e, ids in ex.items():
                out.setdefault(e, []).append((ids, pos[o:o + len(ids)]))
                o += len(ids)
        return out

    def _write_halo_rows(self, parts):
        for part in parts:
            for e, rows in part.items():
                if e not in self.handles:
                    continue
                for ids, pos in rows:
                    if len(ids):
                        call(self.lib, "espp_dd_set_halo_positions", self.handles[e], len(ids),
                             i64ptr(ids), dptr(np.ascontiguousarray(pos)))

    def _refresh_halo_direct(self):
        """The halo refresh in the library's memory space: positions read into a buffer
        on the owner, copied or sent (one message per (owner, holder) pair, posted in
        (owner, holder) order on both sides), written into the holder's halo copies."""
        import torch
        c_i64, c_d = ctypes.c_int64, ctypes.c_double
        sends, recvs = [], []

        def local_part():
            for d in self.local:
                for e, ids in self._xids[d].items():
                    buf = torch.empty(3 * len(ids), dtype=torch.float64, device=ids.device)
                    call(self.lib, "espp_dd_read_positions", self.handles[d], len(ids),
                         self._ptr(ids, c_i64), self._ptr(buf, c_d))
                    if e in self.handles:
                        hid = self._hids[e][d]
                        call(self.lib, "espp_dd_write_halo", self.handles[e], len(hid),
                             self._ptr(hid, c_i64), self._ptr(buf, c_d))
                    else:
                        sends.append((d, e, buf))

        failed = self._guarded(local_part)
        if self.comm.world > 1:
            # every rank learns of a failed read before any point-to-point message
            self._raise_failed(self.comm.allgather(failed))
        elif failed is not None:
            return failed
        for e in self.local:
            for o, hid in self._hids[e].items():
                if o not in self.handles:
                    recvs.append((o, e, hid, torch.empty(3 * len(hid), dtype=torch.float64,
                                                         device=hid.device)))
        if sends or recvs:
            dist = self.comm._dist
            group = self.comm._group
            reqs = [dist.isend(buf, dst=e // self._per, group=group, tag=d * self.D + e)
                    for d, e, buf in sends]
            reqs += [dist.irecv(buf, src=o // self._per, group=group, tag=o * self.D + e)
                     for o, e, _, buf in sorted(recvs, key=lambda r: (r[0], r[1]))]
            for r in reqs:
                r.wait()
            if recvs and recvs[0][3].is_cuda:
                torch.cuda.current_stream().synchronize()

            def write_received():
                for o, e, hid, buf in recvs:
                    call(self.lib, "espp_dd_write_halo", self.handles[e], len(hid),
                         self._ptr(hid, c_i64), self._ptr(buf, c_d))

            return self._guarded(write_received)
        return None

    def _push_bonds(self, e):
        """The bonds with an owned member of domain e; both members must be held."""
        call(self.lib, "espp_bonds_clear", self.handles[e])
        if len(self._bonds) == 0:
            return
        held = np.concatenate([self.owned[e], self.halo[e][0]])
        mine = (np.isin(self._bonds[:, 0], self.owned[e])
                | np.isin(self._bonds[:, 1], self.owned[e]))
        if not np.isin(self._bonds[mine], held).all():
            raise RuntimeError("a bond of domain %d reaches past its halo layer (bond longer "
                               "than halfCellInt cells)" % e)
        b = np.ascontiguousarray(self._bonds[mine]).reshape(-1)
        if len(b):
            call(self.lib, "espp_bonds_add", self.handles[e], len(b) // 2, i64ptr(b))

    # ---- changes of the particle set and state -----------------------------------------
    def replace_particles(self, ids, pos, vel, img, types=None, mass=None):
        """Every rank passes the same whole new set (positions as integrated, images as
        they are); it replaces the particles of all domains, and the next step re-sorts."""
        ids = np.asarray(ids, np.int64)
        n = len(ids)
        if types is not None or mass is not None:
            known = np.isin(ids, self._ids)
            new_ids = ids[~known]
            if len(new_ids):
                t = np.zeros(n, np.int32) if types is None else np.asarray(types, np.int32)
                ms = np.ones(n) if mass is None else np.asarray(mass, np.float64)
                allids = np.concatenate([self._ids, new_ids])
                order = np.argsort(allids, kind="stable")
                self._ids = allids[order]
                self._type = np.concatenate([self._type, t[~known]])[order]
                self._mass = np.concatenate([self._mass, ms[~known]])[order]
        held = (ids, np.array(pos, np.float64).reshape(n, 3),
                np.array(vel, np.float64).reshape(n, 3), np.array(img, np.int32).reshape(n, 3))
        self._load([self._bucket_all(held)])
        keep = np.isin(self._ids, ids)
        self._ids, self._type, self._mass = self._ids[keep], self._type[keep], self._mass[keep]

    def all_particles(self):
        """(ids, pos, vel, img) of every particle, sorted by id, on every rank."""
        parts = self.comm.allgather(self._collect_owned())
        ids = np.concatenate([p[0] for p in parts])
        order = np.argsort(ids)
        return tuple(np.concatenate([p[k] for p in parts])[order] for k in range(4))

    def set_velocities(self, ids, vel):
        ids = np.asarray(ids, np.int64)
        vel = np.asarray(vel, np.float64).reshape(-1, 3)
        for d in self.local:
            sel = np.isin(ids, self.owned[d])
            if sel.any():
                call(self.lib, "espp_set_particles", self.handles[d], int(sel.sum()),
                     i64ptr(np.ascontiguousarray(ids[sel])), None,
                     dptr(np.ascontiguousarray(vel[sel])))

    def set_images(self, ids, img):
        ids = np.asarray(ids, np.int64)
        img = np.asarray(img, np.int32).reshape(-1, 3)
        for d in self.local:
            sel = np.isin(ids, self.owned[d])
            if sel.any():
                call(self.lib, "espp_set_images", self.handles[d], int(sel.sum()),
                     i64ptr(np.ascontiguousarray(ids[sel])),
                     i32ptr(np.ascontiguousarray(img[sel])))

    def set_positions(self, ids, pos):
        """New positions (taken as they are): the particles may change owner, so the set
        is redistributed, and the next step re-sorts."""
        all_ids, p, v, im = self.all_particles()
        k = np.searchsorted(all_ids, np.asarray(ids, np.int64))
        p[k] = np.asarray(pos, np.float64).reshape(-1, 3)
        self.replace_particles(all_ids, p, v, im)

    def step_get(self):
        v = ctypes.c_int64()
        call(self.lib, "espp_step_get", self.handles[self.local[0]], ctypes.byref(v))
        return v.value

    def builds(self):
        out = []
        for d in self.local:
            v = ctypes.c_int64()
            call(self.lib, "espp_vl_builds", self.handles[d], ctypes.byref(v))
            out.append(v.value)
        return int(self._global_max(out))

    # ---- observables ----------------------------------------------------------------
    def _sum(self, values):
        return sum(sum(v) for v in self.comm.allgather(values))

    def _scalar(self, name, *args):
        out = []
        for d in self.local:
            v = ctypes.c_double()
            call(self.lib, name, self.handles[d], *args, ctypes.byref(v))
            out.append(v.value)
        return out

    def energy(self, which):
        return self._sum(self._scalar("espp_energy", int(which)))

    def virial(self, which):
        return self._sum(self._scalar("espp_virial", int(which)))

    def virial_tensor(self, which):
        out = []
        for d in self.local:
            w = np.zeros(6)
            call(self.lib, "espp_virial_tensor", self.handles[d], int(which), dptr(w))
            out.append(w)
        return sum(sum(v) for v in self.comm.allgather(out))

    def kinetic(self):
        """(sum m v^2, number of particles) over the owned particles of all domains."""
        v2, n = [], []
        for d in self.local:
            s = ctypes.c_double()
            k = ctypes.c_int64()
            call(self.lib, "espp_kinetic", self.handles[d], ctypes.byref(s), ctypes.byref(k))
            v2.append(s.value)
            n.append(k.value)
        return self._sum(v2), int(self._sum(n))

    def kinetic_tensor(self):
        out = []
        for d in self.local:
            w = np.zeros(6)
            call(self.lib, "espp_kinetic_tensor", self.handles[d], dptr(w))
            out.append(w)
        return sum(sum(v) for v in self.comm.allgather(out))

    def kinetic_types(self, type_mask):
        v2, n = [], []
        for d in self.local:
            s = ctypes.c_double()
            k = ctypes.c_int64()
            call(self.lib, "espp_kinetic_types", self.handles[d], ctypes.c_uint64(type_mask),
                 ctypes.byref(s), ctypes.byref(k))
            v2.append(s.value)
            n.append(k.value)
        return self._sum(v2), int(self._sum(n))

    def bonds_max_sqr(self):
        """FixedPairList's long-time maximum bond length^2 over all domains."""
        out = []
        for d in self.local:
            v = np.zeros(1)
            call(self.lib, "espp_bonds_max_sqr", self.handles[d], dptr(v))
            out.append(float(v[0]))
        return self._global_max(out)

    def vl_size(self):
        out = []
        for d in self.local:
            n = ctypes.c_int64()
            call(self.lib, "espp_vl_size", self.handles[d], ctypes.byref(n))
            out.append(n.value)
        return int(self._sum(out))

    def vl_pairs(self):
        """Sorted (smaller id, larger id) pairs of the whole system."""
        out = []
        for d in self.local:
            n = ctypes.c_int64()
            call(self.lib, "espp_vl_size", self.handles[d], ctypes.byref(n))
            p = np.zeros(2 * max(n.value, 1), np.int64)
            call(self.lib, "espp_vl_pairs", self.handles[d], n.value, i64ptr(p), ctypes.byref(n))
            out.append(p[:2 * n.value].reshape(-1, 2))
        allp = np.concatenate([p for part in self.comm.allgather(out) for p in part])
        return allp[np.lexsort((allp[:, 1], allp[:, 0]))]

    def vl_digest(self):
        """The pair-set digest of the whole system: counts and sums add, xors combine."""
        out = []
        for d in self.local:
            w = np.zeros(4, np.uint64)
            call(self.lib, "espp_vl_digest", self.handles[d],
                 w.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
            out.append(w)
        t = np.zeros(4, np.uint64)
        with np.errstate(over="ignore"):
            for part in self.comm.allgather(out):
                for w in part:
                    t[0] += w[0]
                    t[1] += w[1]
                    t[2] ^= w[2]
                    t[3] += w[3]
        return tuple(int(x) for x in t)

    def get_particles(self, ids):
        """Positions, velocities, forces and images by id, from the owning domains."""
        ids = np.asarray(ids, np.int64)
        out = []
        for d in self.local:
            sel = ids[np.isin(ids, self.owned[d])]
            if len(sel) == 0:
                continue
            p, v, f = (np.zeros((len(sel), 3)) for _ in range(3))
            im = np.zeros((len(sel), 3), np.int32)
            call(self.lib, "espp_get_particles", self.handles[d], len(sel), i64ptr(sel),
                 dptr(p), dptr(v), dptr(f), i32ptr(im))
            out.append((sel, p, v, f, im))
        rows = [r for part in self.comm.allgather(out) for r in part]
        got = np.concatenate([r[0] for r in rows]) if rows else np.zeros(0, np.int64)
        if len(got) != len(ids) or not np.isin(ids, got).all():
            raise RuntimeError("unknown particle id")
        order = np.argsort(got)
        k = order[np.searchsorted(got[order], ids)]
        return tuple(np.concatenate([r[c] for r in rows])[k] for c in range(1, 5))

    def domain_sizes(self):
        """(owned, halo) particle counts of every domain."""
        out = {}
        for d in self.local:
            n = ctypes.c_int64()
            call(self.lib, "espp_num_particles", self.handles[d], ctypes.byref(n))
            out[d] = (len(self.owned[d]), n.value - len(self.owned[d]))
        res = {}
        for part in self.comm.allgather(out):
            res.update(part)
        return [res[d] for d in range(self.D)]

    def close(self):
        for d in list(self.handles):
            call(self.lib, "espp_system_destroy", self.handles.pop(d))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
