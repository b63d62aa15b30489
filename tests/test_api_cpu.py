"""Host-side pieces of the drop-in API (no GPU): potentials, helpers, tools."""
import math

import pytest

import espressopp_b200 as espressopp


def test_lj_potential_matches_reference_tests():
    lj = espressopp.interaction.LennardJones(1.0, 1.0, espressopp.infinity)
    assert lj.computeEnergy(2 ** (1 / 6)) == pytest.approx(-1.0)
    lj2 = espressopp.interaction.LennardJones(epsilon=2.0, sigma=2.0)
    assert lj2.epsilon == 2.0 and lj2.sigma == 2.0 and math.isinf(lj2.cutoff)
    assert lj2.shift == 0.0
    assert abs(lj2.computeEnergy(2.0)) < 1e-12
    assert lj2.computeEnergy(2 * 2 ** (1 / 6)) == pytest.approx(-2.0)
    assert lj2.computeForce(2 * 2 ** (1 / 6), 0, 0)[0] == pytest.approx(0.0, abs=1e-12)
    lj3 = espressopp.interaction.LennardJones(1.0, 1.0, 2.5)
    assert lj3.shift == pytest.approx(4.0 * (2.5 ** -12 - 2.5 ** -6))
    assert lj3.computeEnergy(2.5) == pytest.approx(0.0, abs=1e-15)
    lj4 = espressopp.interaction.LennardJones(1.0, 1.0, 2.5, shift=0)
    assert lj4.shift == 0.0


def test_fene_potential_matches_reference_tests():
    f = espressopp.interaction.FENE(K=30.0, r0=0.0, rMax=1.5)
    assert f.computeEnergy(0.97) == pytest.approx(18.279, rel=1e-4)
    assert f.computeEnergy(0.80) == pytest.approx(11.296, rel=1e-4)
    assert f.computeEnergy(1.40) == pytest.approx(69.147, rel=1e-4)
    assert list(f.computeForce(0.9, 0.1, 0.1)) == pytest.approx([-42.782, -4.7535, -4.7535],
                                                                rel=1e-4)
    g = espressopp.interaction.FENE(K=1.0, r0=1.0, rMax=0.5)
    assert g.computeEnergy(1.0) == 0.0
    assert g.computeForce(1.0, 0, 0)[0] == 0.0


def test_decomp_cellgrid():
    assert tuple(espressopp.tools.decomp.cellGrid((33.8585,) * 3, (1, 1, 1), 2.5, 0.3)) == (12,) * 3
    assert tuple(espressopp.tools.decomp.cellGrid((36.1033,) * 3, (1, 1, 1), 1.12, 0.3)) == (25,) * 3
    assert tuple(espressopp.tools.decomp.nodeGrid(2, (10,) * 3, 2.5, 0.3)) == (1, 1, 2)
    assert tuple(espressopp.tools.decomp.cellGrid((33.8585,) * 3, (1, 1, 2), 2.5, 0.3)) == (
        12, 12, 6)
    with pytest.raises(ValueError):
        espressopp.tools.decomp.nodeGrid(0)
    # one process without torch.distributed: a world of one
    assert espressopp.MPI.COMM_WORLD.size == 1 and espressopp.MPI.COMM_WORLD.rank == 0


def test_lattice_and_velocities():
    x, y, z, Lx, Ly, Lz = espressopp.tools.lattice.createCubic(1000, 0.8442)
    assert len(x) == 1000 and Lx == pytest.approx((1000 / 0.8442) ** (1 / 3))
    vx, vy, vz = espressopp.tools.velocities.gaussian(1.0, 1000)
    assert abs(sum(vx)) < 1e-9
    T = sum(a * a + b * b + c * c for a, b, c in zip(vx, vy, vz)) / 3000.0
    assert 0.9 < T < 1.1


def test_real3d_and_bc():
    r = espressopp.Real3D(1, 2, 3)
    assert r * r == 14.0 and (r + r)[2] == 6.0 and r.sqr() == 14.0
    rng = espressopp.esutil.RNG(5)
    bc = espressopp.bc.OrthorhombicBC(rng, (10.0, 10.0, 10.0))
    p, img = bc.getFoldedPosition((11.0, -1.0, 5.0))
    assert p == pytest.approx((1.0, 9.0, 5.0)) and tuple(img) == (1, -1, 0)
    for _ in range(10):
        q = bc.getRandomPos()
        assert all(0 <= q[k] < 10 for k in range(3))


def test_precision_selection():
    with pytest.raises(ValueError):
        espressopp.set_default_precision("half")


def test_rng_save_and_load_state(tmp_path, monkeypatch, capsys):
    """RNG.saveState(step) writes rng.<step>; loadState brings the draws back to that
    point (RNG.cpp:86-138), and a file for another number of ranks is refused."""
    monkeypatch.chdir(tmp_path)
    rng = espressopp.esutil.RNG(42)
    [rng() for _ in range(7)]
    rng.saveState(1000)
    after = [rng() for _ in range(5)] + [rng(10), rng.normal()]
    other = espressopp.esutil.RNG(42)
    other.loadState("rng.1000")
    assert [other() for _ in range(5)] + [other(10), other.normal()] == after
    fresh = espressopp.esutil.RNG(7)
    fresh.loadState("rng.1000")
    assert fresh.get_seed() == 42 and fresh() == after[0]
    (tmp_path / "rng.two").write_text(open("rng.1000").read() * 2)
    keep = espressopp.esutil.RNG(3)
    first = espressopp.esutil.RNG(3)()
    keep.loadState("rng.two")
    assert keep.get_seed() == 3 and keep() == first
    assert "number of processes does not match" in capsys.readouterr().err


def test_potentials_pickle():
    """Potentials survive pickling with their parameters (LennardJones_pickle,
    LennardJones.hpp:176-191)."""
    import pickle
    for pot in (espressopp.interaction.LennardJones(1.2, 0.9, 2.5),
                espressopp.interaction.LennardJonesCapped(1.0, 1.0, 2.5, caprad=0.9),
                espressopp.interaction.FENE(K=25.0, r0=0.1, rMax=1.4),
                espressopp.interaction.Cosine(K=1.5, theta0=3.0)):
        q = pickle.loads(pickle.dumps(pot))
        assert type(q) is type(pot) and vars(q) == vars(pot)
    lj = pickle.loads(pickle.dumps(espressopp.interaction.LennardJones(1.2, 0.9, 2.5)))
    assert lj.computeEnergy(2.5) == pytest.approx(0.0, abs=1e-15)


def test_replicate_copies_positions_and_topology():
    """tools.replicate (src/tools/replicate.py): copies in (i, j, k) order, k fastest,
    positions shifted by the box edges, ids by the copy index times N."""
    from espressopp_b200.tools import replicate
    x, y, z = [0.1, 0.2, 0.3], [0.4, 0.5, 0.6], [0.7, 0.8, 0.9]
    b, a, xs, ys, zs, Lx, Ly, Lz = replicate([(1, 2), (2, 3)], [(1, 2, 3)], x, y, z,
                                             1.0, 2.0, 3.0, xdim=2, ydim=1, zdim=2)
    assert (Lx, Ly, Lz) == (2.0, 2.0, 6.0) and len(xs) == 12
    assert xs[3:6] == x and zs[3:6] == [v + 3.0 for v in z]      # copy 1: (0, 0, 1)
    assert xs[6:9] == [v + 1.0 for v in x] and zs[6:9] == z       # copy 2: (1, 0, 0)
    assert b[2:4] == [(4, 5), (5, 6)] and b[-1] == (11, 12)
    assert a == [(1, 2, 3), (4, 5, 6), (7, 8, 9), (10, 11, 12)]
    assert replicate([], [], x, y, z, 1.0, 1.0, 1.0) == ([], [], x, y, z, 1.0, 1.0, 1.0)
    assert espressopp.tools.readxyz is espressopp.tools.DumpConfigurations.readxyz
