"""Every list layout of the GPU path (espp_set_layout) against the FP64 oracle.

Layouts: the global per-particle list (built by runs of 32 particles) with 1, 2, 4 or 8
threads per particle in the force kernel (form 0); the same list built by brick windows (form 2);
brick windows for the build and the force kernels with 16-bit window-index lists (form 1),
for several brick shapes.  For each: the sorted id-pair set equals the oracle's
(VerletList.cpp:274-450), forces agree (FP64 1e-12, mixed 1e-5 relative RMS and 5e-3 of
the RMS force per particle), energy and virial agree to 1e-10 relative, and after steps
that end on a re-sort the list again equals the oracle's at the positions reached.

Systems: an LJ fluid (13,824 particles, 9^3 cells, rc 2.5, skin 0.3), a capped LJ fluid
(the same, cap radius 0.95) and the 40,000-bead ring melt of testsuite/tabulated (WCA +
FENE bonds, bonded pairs excluded from the list).  espp_autotune_layout is run on the LJ
fluid and its choice is checked the same way.
"""
import ctypes
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from espressopp_b200._abi import call, dptr, i32ptr
from simdriver import (Sim, cell_grid, cuda_lib, lattice, load_polymer40k, mb_velocities,
                       oracle_lib)

pytestmark = pytest.mark.gpu

RC, SKIN = 2.5, 0.3
SHIFT = 4.0 * (RC ** -12 - RC ** -6)

LAYOUTS = [(0, 1, (0, 0, 0)), (0, 2, (0, 0, 0)), (0, 4, (0, 0, 0)), (0, 8, (0, 0, 0)),
           (2, 1, (0, 0, 0)), (2, 1, (2, 2, 2)),
           (1, 0, (0, 0, 0)), (1, 0, (1, 2, 2)), (1, 0, (2, 2, 2)), (1, 0, (3, 3, 3))]


def _set_layout(s, form, tpp, brick):
    call(s.lib, "espp_set_layout", s.h, form, tpp, i32ptr(np.asarray(brick, np.int32)))


def _get_layout(s):
    out = np.zeros(5, np.int32)
    call(s.lib, "espp_get_layout", s.h, i32ptr(out))
    return [int(v) for v in out]


def _errors(f, fref):
    df = f - fref
    rms = math.sqrt(np.sum(df * df) / np.sum(fref * fref))
    per = float(np.max(np.linalg.norm(df, axis=1)) /
                math.sqrt(np.mean(np.sum(fref * fref, axis=1))))
    return rms, per


def _lj(lib, prec, ids, pos, vel, box, caprad=0.0):
    s = Sim(lib, box, SKIN, cell_grid(box, RC, SKIN), precision=prec, seed=99)
    s.add(ids, pos, vel)
    s.decompose()
    s.vl(RC)
    s.lj(0, 0, 1.0, 1.0, RC, SHIFT, caprad)
    s.integrator(0.005)
    return s


def _melt(lib, prec, ids, pos, bonds, box):
    s = Sim(lib, box, 0.3, cell_grid(box, 1.12, 0.3), precision=prec, seed=5)
    s.add(ids, pos)
    s.decompose()
    s.vl(1.42, excl=bonds)
    s.lj(0, 0, 1.0, 1.0, 1.12, 0.0)
    s.bonds(bonds)
    s.fene(30.0, 0.0, 1.5)
    s.integrator(0.005)
    return s


def _compare(g, o, ids, prec, which):
    assert g.digest() == o.digest()
    assert np.array_equal(g.pairs(), o.pairs())
    g.run(0)
    rms, per = _errors(g.particles(ids)[2], o.particles(ids)[2])
    if prec == _abi.PREC_FP64:
        assert rms < 1e-12
    else:
        assert rms < 1e-5 and per < 5e-3
    for w in which:
        eo, wo = o.energy(w), o.virial(w)
        assert abs(g.energy(w) - eo) <= 1e-10 * abs(eo)
        assert abs(g.virial(w) - wo) <= 1e-10 * abs(wo)


def _expect_form(g, form):
    got = _get_layout(g)
    assert got[0] == form, got
    if form != 0:
        assert all(b >= 1 for b in got[2:5]), got


def _step_to_resort(g, box, ids, build_oracle, tries=60):
    """Steps until a re-sort happens inside the captured loop, then compares the list in
    use (built at the positions the run ends on) with the oracle's there."""
    for _ in range(tries):
        g.run(1)
        if g.num_resorts() > 0:
            break
    assert g.num_resorts() > 0
    x = g.particles(ids)[0]
    o = build_oracle(x)
    assert g.digest() == o.digest()
    return o


@pytest.fixture(scope="module")
def fluid():
    pos, box = lattice(24, 0.8442, 0.05, 3)
    vel = mb_velocities(len(pos), 1.0, 4)
    ids = np.arange(len(pos), dtype=np.int64)
    assert cell_grid(box, RC, SKIN) == [9, 9, 9]
    o = _lj(oracle_lib(), _abi.PREC_FP64, ids, pos, vel, box)
    o.run(0)
    return ids, pos, vel, box, o


@pytest.mark.parametrize("prec", [_abi.PREC_MIXED, _abi.PREC_FP64])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_lj_fluid_layout(fluid, layout, prec):
    ids, pos, vel, box, o = fluid
    form, tpp, brick = layout
    g = _lj(cuda_lib(), prec, ids, pos, vel, box)
    _set_layout(g, form, tpp, brick)
    _expect_form(g, form)
    if form != 1:
        assert _get_layout(g)[1] == tpp
    if any(brick):
        assert _get_layout(g)[2:5] == list(brick)
    _compare(g, o, ids, prec, [_abi.IA_LJ])

    def at(x):
        oo = _lj(oracle_lib(), _abi.PREC_FP64, ids, x, None, box)
        oo.run(0)
        return oo
    oo = _step_to_resort(g, box, ids, at)
    rms, per = _errors(g.particles(ids)[2], oo.particles(ids)[2])
    assert rms < (1e-12 if prec == _abi.PREC_FP64 else 1e-5)


@pytest.mark.parametrize("layout", [(0, 1, (0, 0, 0)), (1, 0, (2, 2, 2))])
def test_capped_lj_layout(layout):
    pos, box = lattice(24, 0.8442, 0.2, 7)
    ids = np.arange(len(pos), dtype=np.int64)
    o = _lj(oracle_lib(), _abi.PREC_FP64, ids, pos, None, box, caprad=0.95)
    o.run(0)
    g = _lj(cuda_lib(), _abi.PREC_MIXED, ids, pos, None, box, caprad=0.95)
    _set_layout(g, *layout)
    _expect_form(g, layout[0])
    _compare(g, o, ids, _abi.PREC_MIXED, [_abi.IA_LJ])


@pytest.fixture(scope="module")
def melt():
    pos, bonds, box, _ = load_polymer40k()
    ids = np.arange(1, len(pos) + 1, dtype=np.int64)
    o = _melt(oracle_lib(), _abi.PREC_FP64, ids, pos, bonds, box)
    o.run(0)
    return ids, pos, bonds, box, o


@pytest.mark.parametrize("prec", [_abi.PREC_MIXED, _abi.PREC_FP64])
@pytest.mark.parametrize("layout", [(0, 1, (0, 0, 0)), (0, 4, (0, 0, 0)), (2, 1, (0, 0, 0)),
                                    (1, 0, (0, 0, 0)), (1, 0, (2, 3, 3))])
def test_melt_fene_exclusions_layout(melt, layout, prec):
    ids, pos, bonds, box, o = melt
    g = _melt(cuda_lib(), prec, ids, pos, bonds, box)
    _set_layout(g, *layout)
    _expect_form(g, layout[0])
    _compare(g, o, ids, prec, [_abi.IA_LJ, _abi.IA_FENE])
    ex = set(map(tuple, np.sort(bonds, axis=1)))
    assert not ex & set(map(tuple, g.pairs()))


def test_autotune_layout_choice_is_exact(fluid):
    ids, pos, vel, box, o = fluid
    g = _lj(cuda_lib(), _abi.PREC_MIXED, ids, pos, vel, box)
    best = np.zeros(5, np.int32)
    table = np.zeros((32, 8))
    n = ctypes.c_int32()
    call(g.lib, "espp_autotune_layout", g.h, 5.0, i32ptr(best), dptr(table), 32,
         ctypes.byref(n))
    assert n.value >= 6
    rows = table[:n.value]
    assert set(rows[:, 0].astype(int)) == {0, 1, 2}
    assert np.all(rows[:, 5] > 0) and np.all(rows[:, 6] > 0)
    k = int(np.argmin(rows[:, 7]))
    assert int(best[0]) == int(rows[k, 0])
    assert [int(v) for v in best] == _get_layout(g)
    _compare(g, o, ids, _abi.PREC_MIXED, [_abi.IA_LJ])


def test_layout_rejects_bad_arguments(fluid):
    ids, pos, vel, box, _ = fluid
    g = _lj(cuda_lib(), _abi.PREC_MIXED, ids, pos, vel, box)
    for form, tpp, brick in ((3, 1, (0, 0, 0)), (0, 3, (0, 0, 0))):
        with pytest.raises(RuntimeError):
            _set_layout(g, form, tpp, brick)
