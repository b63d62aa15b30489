"""interaction.Tabulated on the host (no GPU): the library's table reader and
interpolation against the oracle's restatement of InterpolationLinear / Akima / Cubic
(src/interaction/Interpolation*.cpp), and the Python mirror."""
import ctypes
import math
import os

import numpy as np
import pytest

from espressopp_b200 import _abi, interaction
from simdriver import cuda_lib, oracle_lib, read_tab, write_tab_file


def _eval(lib, itype, r, e, f, x):
    E = np.zeros(len(x))
    F = np.zeros(len(x))
    _abi.call(lib, "espp_tab_eval", itype, len(r), _abi.dptr(r), _abi.dptr(e), _abi.dptr(f),
              len(x), _abi.dptr(x), _abi.dptr(E), _abi.dptr(F))
    return E, F


@pytest.mark.parametrize("itype", [1, 2, 3])
def test_interpolation_matches_oracle_bitwise(tmp_path, itype):
    lj = interaction.LennardJones(1.0, 1.0, cutoff=2.5)
    path = str(tmp_path / "lj.tab")
    write_tab_file(lj, path, N=301, low=0.8, high=2.5)
    r, e, f = read_tab(cuda_lib(), path)
    r2, e2, f2 = read_tab(oracle_lib(), path)
    assert np.array_equal(r, r2) and np.array_equal(e, e2) and np.array_equal(f, f2)
    rng = np.random.Generator(np.random.PCG64(7))
    x = np.concatenate([rng.uniform(0.8, 2.5, 4000), r, [0.5, 2.5, 3.0]])
    Eg, Fg = _eval(cuda_lib(), itype, r, e, f, x)
    Eo, Fo = _eval(oracle_lib(), itype, r, e, f, x)
    assert np.array_equal(Eg, Eo) and np.array_equal(Fg, Fo)
    inside = (x > 0.85) & (x < 2.45)
    # the tables follow the potential (Akima's reference evaluation keeps only the linear
    # Hermite term, so its error is first order in the spacing)
    tol = {1: 2e-2, 2: 5e-2, 3: 1e-4}[itype]
    Etrue = np.array([lj.computeEnergy(v) for v in x[inside]])
    assert np.max(np.abs(Eg[inside] - Etrue)) < tol * max(1.0, np.max(np.abs(Etrue)))


def test_reader_skips_lines_without_three_numbers(tmp_path):
    path = tmp_path / "t.tab"
    path.write_text("# comment\n0.0 1.0 2.0\n\n1.0 2.0\n0.5 1.5 2.5 extra\nabc 1 2\n1.0 3.0 4.0\n")
    for lib in (cuda_lib(), oracle_lib()):
        r, e, f = read_tab(lib, str(path))
        assert list(r) == [0.0, 0.5, 1.0] and list(e) == [1.0, 1.5, 3.0]
        assert list(f) == [2.0, 2.5, 4.0]


def test_reader_rejects_short_or_missing_files(tmp_path):
    short = tmp_path / "s.tab"
    short.write_text("0.0 1.0 2.0\n")
    for lib in (cuda_lib(), oracle_lib()):
        n = ctypes.c_int64()
        for p in (str(short), str(tmp_path / "missing.tab")):
            rc = lib.espp_tab_read(p.encode(), 0, None, None, None, ctypes.byref(n))
            assert rc == -1


def test_python_tabulated_potential(tmp_path):
    fene = interaction.FENE(K=30.0, r0=0.0, rMax=1.5)
    path = str(tmp_path / "fene.tab")
    write_tab_file(fene, path, N=257, low=0.0001, high=1.49)
    t = interaction.Tabulated(itype=3, filename=path)
    assert t.filename == path and t.itype == 3 and math.isinf(t.cutoff) and t.shift == 0.0
    for rr in (0.5, 0.97, 1.2):
        assert t.computeEnergy(rr) == pytest.approx(fene.computeEnergy(rr), rel=1e-5)
        assert t.computeForce(rr, 0, 0)[0] == pytest.approx(fene.computeForce(rr, 0, 0)[0],
                                                           rel=1e-5)
    tc = interaction.Tabulated(itype=2, filename=path, cutoff=1.0)
    assert tc.computeEnergy(1.1) == 0.0
