"""The C ABI of one system, answered by a spatial decomposition over several domains.

A storage created with a node grid of more than one node (``storage.DomainDecomposition(
system, nodeGrid, cellGrid)`` with nodeGrid from ``tools.decomp.nodeGrid(n)``) holds a
``domain.SpatialDecomposition`` instead of one system handle.  The classes of the Python
mirror call the library as ``call(storage._lib, "espp_...", storage._h, ...)``; this
module's ``DecomposedLibrary`` stands in for the library there: each entry point the
mirror uses is forwarded to every domain (settings), to the owning domains (particle
state), or summed over the domains (observables).  Entry points that need the whole
system in one place (angles, the RDF, configurations, the learned potential) raise an
error naming the limitation.
"""
import numpy as np

from . import _abi


def _arr(ptr, shape, dtype):
    """A numpy view of a ctypes pointer argument (None stays None)."""
    if ptr is None:
        return None
    a = np.ctypeslib.as_array(ptr, shape=shape)
    assert a.dtype == np.dtype(dtype)
    return a


def _out(ref, value):
    """Stores value through a ctypes.byref argument."""
    ref._obj.value = value


class DecomposedLibrary:
    """Stands in for the loaded C ABI library behind a decomposed storage."""

    def __init__(self, sd):
        self.sd = sd
        self._lib = sd.lib

    def __getattr__(self, name):
        if name.startswith("espp_"):
            def refuse(*args):
                raise RuntimeError("%s is not available on a storage decomposed over several "
                                   "nodes (it needs the whole system in one place)" % name)
            return refuse
        raise AttributeError(name)

    # handle-free entry points go to the library itself
    def espp_tab_read(self, *args):
        return self._lib.espp_tab_read(*args)

    def espp_tab_eval(self, *args):
        return self._lib.espp_tab_eval(*args)

    def espp_last_error(self, *args):
        return self._lib.espp_last_error(*args)

    def espp_system_destroy(self, h):
        self.sd.close()
        return 0

    # ---- settings: every domain ----------------------------------------------------
    def _each(self, name, *args):
        for d in self.sd.local:
            _abi.call(self._lib, name, self.sd.handles[d], *args)
        return 0

    def espp_set_skin(self, h, skin):
        self.sd.skin = float(skin)
        return self._each("espp_set_skin", skin)

    def espp_vl_create(self, h, cutoff, nexcl, excl):
        return self._each("espp_vl_create", cutoff, nexcl, excl)

    def espp_vl_rebuild(self, h):
        return self._each("espp_vl_rebuild")

    def espp_lj_set(self, h, *args):
        return self._each("espp_lj_set", *args)

    def espp_fene_set(self, h, *args):
        return self._each("espp_fene_set", *args)

    def espp_tab_pair_set(self, h, *args):
        return self._each("espp_tab_pair_set", *args)

    def espp_tab_bond_set(self, h, *args):
        return self._each("espp_tab_bond_set", *args)

    def espp_integrator_set(self, h, dt):
        return self._each("espp_integrator_set", dt)

    def espp_step_set(self, h, step):
        return self._each("espp_step_set", step)

    def espp_langevin_set(self, h, *args):
        return self._each("espp_langevin_set", *args)

    def espp_capforce_set(self, h, *args):
        return self._each("espp_capforce_set", *args)

    def espp_bonds_reset_max(self, h):
        return self._each("espp_bonds_reset_max")

    # ---- particles -------------------------------------------------------------------
    def espp_add_particles(self, h, n, ids, typ, mass, pos, vel):
        n = int(n)
        self.sd.add_particles(_arr(ids, (n,), np.int64).copy(),
                              _arr(pos, (3 * n,), np.float64).reshape(n, 3),
                              None if vel is None else _arr(vel, (3 * n,), np.float64),
                              None if typ is None else _arr(typ, (n,), np.int32).copy(),
                              None if mass is None else _arr(mass, (n,), np.float64).copy())
        return 0

    def espp_decompose(self, h):
        self.sd.decompose()
        return 0

    def espp_get_particles(self, h, n, ids, pos, vel, force, img):
        n = int(n)
        p, v, f, im = self.sd.get_particles(_arr(ids, (n,), np.int64))
        for ptr, val, dt in ((pos, p, np.float64), (vel, v, np.float64),
                             (force, f, np.float64), (img, im, np.int32)):
            if ptr is not None:
                _arr(ptr, (3 * n,), dt)[:] = val.reshape(-1)
        return 0

    def espp_set_particles(self, h, n, ids, pos, vel):
        n = int(n)
        i = _arr(ids, (n,), np.int64).copy()
        if vel is not None:
            self.sd.set_velocities(i, _arr(vel, (3 * n,), np.float64).copy())
        if pos is not None:
            self.sd.set_positions(i, _arr(pos, (3 * n,), np.float64).copy())
        return 0

    def espp_set_images(self, h, n, ids, img):
        n = int(n)
        self.sd.set_images(_arr(ids, (n,), np.int64).copy(), _arr(img, (3 * n,), np.int32).copy())
        return 0

    def espp_dd_load(self, h, n, ids, typ, mass, pos, vel, img, halo):
        """The mirror's particle removal: the given set replaces all particles."""
        n = int(n)
        self.sd.replace_particles(
            _arr(ids, (n,), np.int64).copy() if n else np.zeros(0, np.int64),
            _arr(pos, (3 * n,), np.float64).copy() if n else np.zeros(0),
            _arr(vel, (3 * n,), np.float64).copy() if n else np.zeros(0),
            _arr(img, (3 * n,), np.int32).copy() if n else np.zeros(0, np.int32))
        return 0

    def espp_bonds_add(self, h, n, pairs):
        n = int(n)
        self.sd.bonds_add(_arr(pairs, (2 * n,), np.int64).copy().reshape(n, 2))
        return 0

    def espp_bonds_clear(self, h):
        self.sd._bonds = np.zeros((0, 2), np.int64)
        for d in self.sd.local:
            self.sd._push_bonds(d)
        return 0

    # ---- the step loop ---------------------------------------------------------------
    def espp_run(self, h, nsteps):
        self.sd.run(int(nsteps))
        return 0

    def espp_num_resorts(self, h, out):
        _out(out, self.sd.last_resorts)
        return 0

    def espp_step_get(self, h, out):
        _out(out, self.sd.step_get())
        return 0

    def espp_vl_builds(self, h, out):
        _out(out, self.sd.builds())
        return 0

    def espp_timers(self, h, t):
        tt = np.zeros(10)
        for d in self.sd.local:
            w = np.zeros(10)
            _abi.call(self._lib, "espp_timers", self.sd.handles[d], _abi.dptr(w))
            tt = np.maximum(tt, w)
        _arr(t, (10,), np.float64)[:] = tt
        return 0

    # ---- observables: summed over the domains ---------------------------------------
    def espp_energy(self, h, which, out):
        _out(out, self.sd.energy(int(which)))
        return 0

    def espp_virial(self, h, which, out):
        _out(out, self.sd.virial(int(which)))
        return 0

    def espp_virial_tensor(self, h, which, w):
        _arr(w, (6,), np.float64)[:] = self.sd.virial_tensor(int(which))
        return 0

    def espp_kinetic(self, h, sum_mv2, n):
        v2, k = self.sd.kinetic()
        _out(sum_mv2, v2)
        _out(n, k)
        return 0

    def espp_kinetic_tensor(self, h, w):
        _arr(w, (6,), np.float64)[:] = self.sd.kinetic_tensor()
        return 0

    def espp_kinetic_types(self, h, mask, sum_mv2, n):
        v2, k = self.sd.kinetic_types(int(mask.value if hasattr(mask, "value") else mask))
        _out(sum_mv2, v2)
        _out(n, k)
        return 0

    def espp_vl_size(self, h, out):
        _out(out, self.sd.vl_size())
        return 0

    def espp_vl_pairs(self, h, cap, pairs, npairs):
        p = self.sd.vl_pairs()
        m = min(int(cap), len(p))
        if m:
            _arr(pairs, (2 * m,), np.int64)[:] = p[:m].reshape(-1)
        _out(npairs, len(p))
        return 0

    def espp_bonds_max_sqr(self, h, out):
        v = self.sd.bonds_max_sqr()
        if hasattr(out, "_obj"):
            _out(out, v)
        else:
            _arr(out, (1,), np.float64)[0] = v
        return 0
