"""espp_energy_noalloc against espp_energy, through the C ABI on the GPU.

Some callers may not allocate GPU memory or have a library allocate it for them: their
device memory belongs to another allocator (a framework's pool or caching allocator,
or a fixed budget), or a first-use cudaMalloc would stall a time-critical loop.
espp_energy_noalloc serves them from a fixed scratch array inside the library
(at most 8,388,608 particles).  It must give the energies of espp_energy, call after
call, whether it runs first in a fresh process or after every other test.
"""
import ctypes

import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import Sim, cell_grid, cuda_lib, load_lj2048, load_polymer40k

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12


def _noalloc(sim, which):
    v = ctypes.c_double()
    _abi.call(sim.lib, "espp_energy_noalloc", sim.h, which, ctypes.byref(v))
    return v.value


def _close(a, b):
    return abs(a - b) <= REL_TOL * max(abs(b), 1.0)


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_noalloc_lj_energy_matches_energy(prec):
    pid, pos, vel, box = load_lj2048()
    s = Sim(cuda_lib(), box, 0.3, cell_grid(box, 2.5, 0.3), precision=prec)
    s.add(pid, pos, vel)
    s.decompose()
    s.vl(2.5)
    s.lj(0, 0, 1.0, 1.0, 2.5, 4.0 * (2.5 ** -12 - 2.5 ** -6))
    ref = s.energy(_abi.IA_LJ)
    assert ref < 0.0
    for _ in range(2):
        assert _close(_noalloc(s, _abi.IA_LJ), ref)
    s.integrator(0.005)
    s.run(25)  # positions change, at least one re-sort
    ref2 = s.energy(_abi.IA_LJ)
    assert ref2 != ref
    for _ in range(2):
        assert _close(_noalloc(s, _abi.IA_LJ), ref2)


def test_noalloc_polymer_melt_lj_and_fene():
    pos, bonds, box, gold = load_polymer40k()
    s = Sim(cuda_lib(), box, 0.3, cell_grid(box, 1.12, 0.3), precision=_abi.PREC_MIXED)
    s.add(np.arange(1, len(pos) + 1), pos)
    s.decompose()
    s.vl(1.42)
    s.lj(0, 0, 1.0, 1.0, 1.12, 0.0)
    s.bonds(bonds)
    s.fene(30.0, 0.0, 1.5)
    for which, golden in ((_abi.IA_LJ, gold["epair"]), (_abi.IA_FENE, gold["ebond"])):
        ref = s.energy(which)
        for _ in range(2):
            got = _noalloc(s, which)
            assert _close(got, ref)
            assert round(got, 3) == golden


def test_noalloc_rejects_unready_system():
    pid, pos, vel, box = load_lj2048()
    s = Sim(cuda_lib(), box, 0.3, cell_grid(box, 2.5, 0.3))
    s.add(pid, pos, vel)  # not sorted yet: the call must refuse instead of building
    v = ctypes.c_double()
    rc = s.lib.espp_energy_noalloc(s.h, _abi.IA_LJ, ctypes.byref(v))
    assert rc == -2
    assert "Verlet list" in _abi.last_error(s.lib)
