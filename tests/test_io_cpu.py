"""io.DumpXYZ (src/io/DumpXYZ.cpp:43-106) frame format, backup of an existing file
(src/io/FileBackup.hpp:37-70), and a round trip through tools.readxyz."""
import os

import numpy as np

from espressopp_b200 import io
from espressopp_b200.tools import DumpConfigurations


class _Storage:
    def __init__(self, ids, pos, vel, img, types):
        self._types = {int(i): int(t) for i, t in zip(ids, types)}
        self._all = (np.asarray(ids), np.asarray(pos, float), np.asarray(vel, float),
                     np.zeros((len(ids), 3)), np.asarray(img))

    def getAll(self):
        return self._all


class _BC:
    boxL = (10.0, 12.5, 8.0)


class _System:
    def __init__(self, st):
        self.storage = st
        self.bc = _BC()


class _Integrator:
    step = 42


def _system():
    ids = [3, 7, 11]
    pos = [[1.0, 2.0, 3.0], [9.5, 0.25, 7.75], [4.125, 11.0, 0.5]]
    vel = [[0.1, -0.2, 0.3], [0.0, 0.5, -0.5], [1.25, 0.0, 0.0]]
    img = [[0, 0, 0], [1, -1, 0], [0, 0, 2]]
    return _System(_Storage(ids, pos, vel, img, [0, 1, 0])), ids, pos, vel, img


def test_dumpxyz_frame_format(tmp_path):
    sysm, ids, pos, vel, img = _system()
    path = str(tmp_path / "traj.xyz")
    d = io.DumpXYZ(sysm, _Integrator(), filename=path, store_pids=True, store_velocities=True)
    d.dump()
    d.dump()
    lines = open(path).read().splitlines()
    assert len(lines) == 2 * (2 + 3)
    assert lines[0] == "3"
    assert lines[1] == "10  0.0  0.0  0.0  12.5  0.0  0.0  0.0  8  currentStep 42  lengthUnit LJ"
    assert lines[2] == "3 0 1.0000000000 2.0000000000 3.0000000000 0.1000000000 -0.2000000000 " \
                       "0.3000000000"
    assert lines[3].startswith("7 1 9.5000000000 0.2500000000 7.7500000000")
    # unfolded positions, scaled lengths, no ids or velocities
    path2 = str(tmp_path / "u.xyz")
    io.DumpXYZ(sysm, _Integrator(), filename=path2, unfolded=True, length_factor=2.0,
               length_unit="nm").dump()
    l2 = open(path2).read().splitlines()
    assert l2[1] == "20  0.0  0.0  0.0  25  0.0  0.0  0.0  16  currentStep 42  lengthUnit nm"
    x = np.array(pos[1]) + np.array(img[1]) * np.array(_BC.boxL)
    assert l2[3] == "1 %.10f %.10f %.10f" % tuple(2.0 * x)


def test_dumpxyz_backup_and_readxyz_round_trip(tmp_path, monkeypatch):
    sysm, ids, pos, vel, img = _system()
    monkeypatch.chdir(tmp_path)
    with open("state.xyz", "w") as f:
        f.write("old\n")
    io.DumpXYZ(sysm, _Integrator(), filename="state.xyz", store_pids=True,
               store_velocities=True, append=False).dump()
    backups = [n for n in os.listdir(tmp_path) if n.endswith("_state.xyz")]
    assert len(backups) == 1 and open(backups[0]).read() == "old\n"
    pid, typ, xp, yp, zp, xv, yv, zv, Lx, Ly, Lz = DumpConfigurations.readxyz("state.xyz")
    assert pid == ids and typ == [0, 1, 0]
    assert np.allclose(np.c_[xp, yp, zp], pos, atol=1e-10)
    assert np.allclose(np.c_[xv, yv, zv], vel, atol=1e-10)
    assert (Lx, Ly, Lz) == (10.0, 12.5, 8.0)


def _lammps_file(path, natoms, nbonds, nangles, ndih, ntypes, velocities=False):
    lines = ["LAMMPS data file", "",
             "%d atoms" % natoms, "%d bonds" % nbonds, "%d angles" % nangles,
             "%d dihedrals" % ndih, "0 impropers", "",
             "%d atom types%s" % (ntypes, " velocities" if velocities else ""), "",
             "0.0 10.0 xlo xhi", "-1.0 11.0 ylo yhi", "2.0 14.0 zlo zhi", "", "Atoms", ""]
    for i in range(natoms):
        if ntypes == 1:
            mol = ["1"] if nbonds else []
            lines.append(" ".join([str(i + 1)] + mol + ["1", "%g" % (i + 0.5), "%g" % (i + 1.5),
                                                        "%g" % (i + 2.5)]))
        else:
            lines.append("%d 1 %d %g %g %g %g" % (i + 1, i % 2, 0.5 * i, i + 0.5, i + 1.5,
                                                  i + 2.5))
    for name, n, width in (("Bonds", nbonds, 2), ("Angles", nangles, 3),
                           ("Dihedrals", ndih, 4)):
        if n:
            lines += ["", name, ""]
            for k in range(n):
                lines.append(" ".join(map(str, [k + 1, 1] + [k + 1 + j for j in range(width)])))
    if velocities:
        lines += ["", "Velocities", ""]
        for i in range(natoms):
            lines.append("%d %g %g %g" % (i + 1, 0.1 * i, -0.1 * i, 0.2))
    path.write_text("\n".join(lines) + "\n")
    return str(path)


def test_lammps_read_return_shapes(tmp_path):
    """tools.lammps.read returns what the reference returns for each kind of file
    (src/tools/lammps.py:142-155)."""
    from espressopp_b200.tools import lammps
    r = lammps.read(_lammps_file(tmp_path / "a.data", 3, 0, 0, 0, 1))
    assert len(r) == 6 and r[0] == [0.5, 1.5, 2.5] and r[3:] == (10.0, 12.0, 12.0)
    r = lammps.read(_lammps_file(tmp_path / "v.data", 3, 0, 0, 0, 1, velocities=True))
    assert len(r) == 9 and r[6] == [0.0, 0.1, 0.2] and r[8] == [0.2] * 3
    r = lammps.read(_lammps_file(tmp_path / "b.data", 4, 3, 0, 0, 1))
    assert len(r) == 7 and r[0] == [(1, 2), (2, 3), (3, 4)] and r[1] == [0.5, 1.5, 2.5, 3.5]
    r = lammps.read(_lammps_file(tmp_path / "ba.data", 4, 3, 2, 0, 1))
    assert len(r) == 8 and r[1] == [(1, 2, 3), (2, 3, 4)] and r[4] == [2.5, 3.5, 4.5, 5.5]
    r = lammps.read(_lammps_file(tmp_path / "bad.data", 5, 4, 3, 2, 1))
    assert len(r) == 9 and r[2] == [(1, 2, 3, 4), (2, 3, 4, 5)]
    r = lammps.read(_lammps_file(tmp_path / "t.data", 4, 3, 2, 0, 2))
    p_type, bonds, angles, q, x, y, z, Lx, Ly, Lz = r
    assert p_type == [0, 1, 0, 1] and q == [0.0, 0.5, 1.0, 1.5] and x[3] == 3.5
    assert bonds == [(1, 2), (2, 3), (3, 4)] and (Lx, Ly, Lz) == (10.0, 12.0, 12.0)
