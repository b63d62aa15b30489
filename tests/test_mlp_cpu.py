"""The learned coarse-grained potential in the FP64 oracle: analytic forces against
finite differences of the energy, and the analytic force-matching gradient against
finite differences of the loss (CPU only)."""
import ctypes
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import Sim, cell_grid, cuda_lib, oracle_lib

NP = 64 * 16 + 64 + 64 * 64 + 64 + 64 + 1


def make_model(lib, seed=1, rc=3.0):
    m = ctypes.c_void_p()
    _abi.call(lib, "espp_mlp_create", rc, 0.0, ctypes.byref(m))
    rng = np.random.Generator(np.random.PCG64(seed))
    theta = np.concatenate([rng.normal(0, 0.25, 64 * 16), rng.normal(0, 0.1, 64),
                            rng.normal(0, 0.125, 64 * 64), rng.normal(0, 0.1, 64),
                            rng.normal(0, 0.125, 64), [0.3]])
    _abi.call(lib, "espp_mlp_set_params", m, NP, _abi.dptr(theta))
    shift = np.full(16, 0.5)
    scale = np.full(16, 0.8)
    _abi.call(lib, "espp_mlp_set_norm", m, _abi.dptr(shift), _abi.dptr(scale))
    _abi.call(lib, "espp_mlp_set_mode", m, 0)  # FP32 site network: strict parity checks
    return m, theta


def cg_system(lib, n=120, seed=2, rho=0.21, rc=3.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    L = (n / rho) ** (1 / 3)
    # well-separated random sites: minimum distance 0.7
    pos = []
    while len(pos) < n:
        p = rng.uniform(0, L, 3)
        if all(np.linalg.norm((p - q) - L * np.round((p - q) / L)) > 0.7 for q in pos):
            pos.append(p)
    pos = np.array(pos)
    box = np.array([L, L, L])
    s = Sim(lib, box, 0.3, cell_grid(box, rc, 0.3))
    s.add(np.arange(1, n + 1), pos, np.zeros_like(pos))
    s.decompose()
    s.vl(rc)
    return s, pos, box


def test_oracle_forces_are_minus_energy_gradient():
    lib = oracle_lib()
    s, pos, box = cg_system(lib)
    m, _ = make_model(lib)
    _abi.call(lib, "espp_mlp_attach", s.h, m)
    s.integrator(0.001)
    s.run(0)
    ids = np.arange(1, len(pos) + 1)
    f = s.particles(ids)[2]
    h = 1e-6

    def energy_at(p):
        _abi.call(lib, "espp_set_particles", s.h, len(ids), _abi.i64ptr(ids),
                  _abi.dptr(np.ascontiguousarray(p.reshape(-1))), None)
        return s.energy(_abi.IA_MLP)

    for a in (0, 7, 55):
        for c in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[a, c] += h
            pm[a, c] -= h
            fd = -(energy_at(pp) - energy_at(pm)) / (2 * h)
            assert fd == pytest.approx(f[a, c], rel=1e-5, abs=1e-7)
    _abi.call(lib, "espp_set_particles", s.h, len(ids), _abi.i64ptr(ids),
              _abi.dptr(np.ascontiguousarray(pos.reshape(-1))), None)
    _abi.call(lib, "espp_mlp_destroy", m)


def test_oracle_force_matching_gradient_matches_finite_differences():
    lib = oracle_lib()
    s, pos, box = cg_system(lib, n=90)
    m, theta = make_model(lib, seed=3)
    _abi.call(lib, "espp_mlp_attach", s.h, m)
    ids = np.arange(1, len(pos) + 1)
    rng = np.random.Generator(np.random.PCG64(9))
    fref = rng.normal(0, 1.0, (len(ids), 3))
    grad = np.zeros(NP)
    loss = ctypes.c_double()
    _abi.call(lib, "espp_mlp_fm_grad", s.h, len(ids), _abi.i64ptr(ids),
              _abi.dptr(np.ascontiguousarray(fref.reshape(-1))), ctypes.byref(loss),
              _abi.dptr(grad))
    h = 1e-6
    check = [0, 5, 64 * 16 + 3, 64 * 16 + 64 + 100, 64 * 16 + 64 + 64 * 64 + 7,
             64 * 16 + 64 + 64 * 64 + 64 + 11, NP - 1, 500, 3000]
    for q in check:
        vals = []
        for sgn in (1, -1):
            t = theta.copy()
            t[q] += sgn * h
            _abi.call(lib, "espp_mlp_set_params", m, NP, _abi.dptr(t))
            l = ctypes.c_double()
            _abi.call(lib, "espp_mlp_fm_grad", s.h, len(ids), _abi.i64ptr(ids),
                      _abi.dptr(np.ascontiguousarray(fref.reshape(-1))), ctypes.byref(l), None)
            vals.append(l.value)
        fd = (vals[0] - vals[1]) / (2 * h)
        assert grad[q] == pytest.approx(fd, rel=1e-4, abs=1e-9), q
    _abi.call(lib, "espp_mlp_destroy", m)
