"""The learned coarse-grained potential on the GPU against the FP64 oracle:
descriptors, site energies, forces (both precision modes), the force-matching loss and
gradient, and training / MD on the GPU."""
import ctypes
import math

import numpy as np
import pytest

from espressopp_b200 import _abi
from simdriver import Sim, cell_grid, cuda_lib, lattice, oracle_lib
from test_mlp_cpu import NP, cg_system, make_model

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def _pair(n=400, seed=2, prec=_abi.PREC_FP64):
    out = []
    for lib, p in ((oracle_lib(), _abi.PREC_FP64), (cuda_lib(), prec)):
        s, pos, box = cg_system(lib, n=n, seed=seed)
        if lib is cuda_lib() and prec != _abi.PREC_FP64:
            s = Sim(lib, box, 0.3, cell_grid(box, 3.0, 0.3), precision=prec)
            s.add(np.arange(1, n + 1), pos, np.zeros_like(pos))
            s.decompose()
            s.vl(3.0)
        m, theta = make_model(lib, seed=5)
        _abi.call(lib, "espp_mlp_attach", s.h, m)
        out.append((s, m))
    return out, pos


@pytest.mark.parametrize("prec", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_mlp_descriptors_energy_forces_match_oracle(prec):
    ((o, mo), (g, mg)), pos = _pair(prec=prec)
    ids = np.arange(1, len(pos) + 1)
    Go, Gg = np.zeros((len(ids), 16)), np.zeros((len(ids), 16))
    _abi.call(o.lib, "espp_mlp_descriptors", o.h, len(ids), _abi.i64ptr(ids), _abi.dptr(Go))
    _abi.call(g.lib, "espp_mlp_descriptors", g.h, len(ids), _abi.i64ptr(ids), _abi.dptr(Gg))
    assert _rel(Gg, Go) < 1e-5
    eo, eg = o.energy(_abi.IA_MLP), g.energy(_abi.IA_MLP)
    assert abs(eg - eo) < 1e-5 * abs(eo)
    for s in (o, g):
        s.integrator(0.002)
        s.run(0)
    assert _rel(g.particles(ids)[2], o.particles(ids)[2]) < 1e-4


def test_mlp_force_matching_gradient_matches_oracle():
    (o, mo), (g, mg) = _pair()[0]
    ids = np.arange(1, 401)
    rng = np.random.Generator(np.random.PCG64(4))
    fref = np.ascontiguousarray(rng.normal(0, 1.0, (400, 3)).reshape(-1))
    go, gg = np.zeros(NP), np.zeros(NP)
    lo, lg = ctypes.c_double(), ctypes.c_double()
    _abi.call(o.lib, "espp_mlp_fm_grad", o.h, 400, _abi.i64ptr(ids), _abi.dptr(fref),
              ctypes.byref(lo), _abi.dptr(go))
    _abi.call(g.lib, "espp_mlp_fm_grad", g.h, 400, _abi.i64ptr(ids), _abi.dptr(fref),
              ctypes.byref(lg), _abi.dptr(gg))
    assert lg.value == pytest.approx(lo.value, rel=1e-5)
    assert _rel(gg, go) < 1e-3
    # each weight block separately (W1, b1, W2, b2, w3)
    for a, b in ((0, 1024), (1024, 1088), (1088, 5184), (5184, 5248), (5248, 5312)):
        assert _rel(gg[a:b], go[a:b]) < 2e-3


def _lattice_pair(n_side):
    """CG-like sites on a jittered simple-cubic lattice at density 0.21 (both libraries)."""
    pos, box = lattice(n_side, 0.21, 0.3, 11)
    out = []
    for lib in (oracle_lib(), cuda_lib()):
        s = Sim(lib, box, 0.3, cell_grid(box, 3.0, 0.3))
        s.add(np.arange(1, len(pos) + 1), pos, np.zeros_like(pos))
        s.decompose()
        s.vl(3.0)
        m, _ = make_model(lib, seed=5)
        _abi.call(lib, "espp_mlp_attach", s.h, m)
        out.append((s, m))
    return out, len(pos)


@pytest.mark.parametrize("n_side", [0, 27])
def test_mlp_tensor_core_gradient_matches_oracle(n_side):
    """The force-matching gradient with its matrix products on the tensor cores (BF16
    operands, FP32 accumulation; espp_mlp_set_mode 1) against the FP64 oracle and the
    FP32 CUDA-core gradient: the BF16 rounding of the operands leaves a few 1e-3 relative
    per weight block.  400 random sites fill part of one 128-site tile per CTA; 27^3 =
    19,683 lattice sites give every CTA several tiles, so the accumulators carry over
    tiles."""
    if n_side:
        ((o, mo), (g, mg)), nsites = _lattice_pair(n_side)
    else:
        nsites = 400
        (o, mo), (g, mg) = _pair(n=nsites)[0]
    ids = np.arange(1, nsites + 1)
    rng = np.random.Generator(np.random.PCG64(4))
    fref = np.ascontiguousarray(rng.normal(0, 1.0, (nsites, 3)).reshape(-1))
    go = np.zeros(NP)
    lo = ctypes.c_double()
    _abi.call(o.lib, "espp_mlp_fm_grad", o.h, nsites, _abi.i64ptr(ids), _abi.dptr(fref),
              ctypes.byref(lo), _abi.dptr(go))
    res = {}
    for mode in (0, 1):
        _abi.call(g.lib, "espp_mlp_set_mode", mg, mode)
        gg = np.zeros(NP)
        lg = ctypes.c_double()
        _abi.call(g.lib, "espp_mlp_fm_grad", g.h, nsites, _abi.i64ptr(ids), _abi.dptr(fref),
                  ctypes.byref(lg), _abi.dptr(gg))
        res[mode] = gg
    _abi.call(g.lib, "espp_mlp_set_mode", mg, 0)
    assert _rel(res[0], go) < 1e-3
    assert _rel(res[1], go) < 2e-2
    for a, b in ((0, 1024), (1024, 1088), (1088, 5184), (5184, 5248), (5248, 5312)):
        assert _rel(res[1][a:b], go[a:b]) < 3e-2
    # the direction that Adam follows
    cos = float(np.dot(res[1], go) / (np.linalg.norm(res[1]) * np.linalg.norm(go)))
    assert cos > 0.999


def test_mlp_training_lowers_the_loss_and_md_runs():
    """A few Adam steps on the GPU fit forces of a known smooth pair potential; then the
    trained model drives NVE dynamics with bounded energy drift."""
    lib = cuda_lib()
    s, pos, box = cg_system(lib, n=400, seed=6)
    ids = np.arange(1, 401)
    # reference forces from a soft tabulated-like pair potential evaluated by the oracle
    o, _, _ = cg_system(oracle_lib(), n=400, seed=6)
    o.lj(0, 0, 0.2, 0.6, 3.0, 4 * 0.2 * ((0.6 / 3.0) ** 12 - (0.6 / 3.0) ** 6))
    o.integrator(0.001)
    o.run(0)
    fref = np.ascontiguousarray(o.particles(ids)[2].reshape(-1))
    m, _ = make_model(lib, seed=7)
    _abi.call(lib, "espp_mlp_attach", s.h, m)
    losses = []
    for it in range(60):
        l = ctypes.c_double()
        _abi.call(lib, "espp_mlp_fm_grad", s.h, 400, _abi.i64ptr(ids), _abi.dptr(fref),
                  ctypes.byref(l), None)
        _abi.call(lib, "espp_mlp_adam_step", m, 3e-3, 0.9, 0.999, 1e-8, 1.0)
        losses.append(l.value)
    assert losses[-1] < 0.5 * losses[0]
    s.integrator(0.002)
    s.run(0)
    e0 = s.energy(_abi.IA_MLP) + 0.5 * s.kinetic()[0]
    s.run(200)
    e1 = s.energy(_abi.IA_MLP) + 0.5 * s.kinetic()[0]
    assert math.isfinite(e1) and abs(e1 - e0) / 400 < 1e-3
    _abi.call(lib, "espp_mlp_destroy", m)


def test_mlp_tensor_core_site_network_matches_fp32():
    """BF16 tcgen05 site network against the FP32 CUDA-core one on the same configuration
    (1,000 sites: eight 128-site tiles, the last one partial) and against the oracle."""
    lib = cuda_lib()
    s, pos, box = cg_system(lib, n=1000, seed=8)
    o, _, _ = cg_system(oracle_lib(), n=1000, seed=8)
    m, _ = make_model(lib, seed=9)
    mo, _ = make_model(oracle_lib(), seed=9)
    _abi.call(lib, "espp_mlp_attach", s.h, m)
    _abi.call(o.lib, "espp_mlp_attach", o.h, mo)
    ids = np.arange(1, 1001)
    res = {}
    for mode in (0, 1):
        _abi.call(lib, "espp_mlp_set_mode", m, mode)
        s.integrator(0.002)
        s.run(0)
        res[mode] = (s.energy(_abi.IA_MLP), s.particles(ids)[2])
    o.integrator(0.002)
    o.run(0)
    eo, fo = o.energy(_abi.IA_MLP), o.particles(ids)[2]
    assert abs(res[0][0] - eo) < 1e-5 * abs(eo)
    # BF16 operands: a few 1e-3 relative in energy and forces
    assert abs(res[1][0] - eo) < 2e-2 * abs(eo)
    assert _rel(res[1][1], fo) < 3e-2
    assert _rel(res[1][1], res[0][1]) < 3e-2
    _abi.call(lib, "espp_mlp_destroy", m)
