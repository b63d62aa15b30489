"""Regenerates the golden fixtures in this directory from the ESPResSo++ test suite.

Run with the path of an ESPResSo++ source tree, given as the argument or in the
environment variable ESPRESSOPP_SRC:

    python tests/golden/make_golden.py REFERENCE_ROOT

Outputs (all committed; nothing at test time reads the reference tree):

* ``lj_fluid_2048.npz`` - the 2048-particle LJ fluid of
  ``testsuite/verlet_list_buffer/lennard_jones_fluid_10000.xyz`` (box 13.4367695311,
  density 0.8442, with velocities), parsed the way ``tools.readxyz``
  (src/tools/DumpConfigurations.py:103-145) parses it.
* ``polymer_melt_40k.npz`` - the 40 000-bead ring melt of
  ``testsuite/tabulated/polymer_melt.start`` (LAMMPS data, parsed like
  ``tools.lammps.read``, src/tools/lammps.py:33-120).  Coordinates have three decimals
  in the file, so they are stored exactly as int32 thousandths; ``x / 1000.0`` rebuilds
  the same doubles Python's ``float()`` gives for the text.
* ``polymer_melt_40k.json`` - the step-0 observables printed in
  ``testsuite/tabulated/result.dat`` for that configuration (LJ rc=1.12 shift 0,
  FENE K=30 r0=0 rMax=1.5, Cosine K=1.5; Verlet cutoff 1.42 + skin 0.3).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_xyz(path):
    with open(path) as f:
        n = int(f.readline().split()[0])
        box = [float(v) for v in f.readline().split()]
        if len(box) != 3:
            box = [box[0], box[4], box[8]]
        pid, typ, pos, vel = [], [], [], []
        for _ in range(n):
            t = f.readline().split()
            if len(t) in (4, 7):
                t.insert(1, "0")
            pid.append(int(t[0]))
            typ.append(int(t[1]))
            pos.append([float(t[2]), float(t[3]), float(t[4])])
            vel.append([float(t[5]), float(t[6]), float(t[7])] if len(t) > 5 else [0.0] * 3)
    return (np.array(pid, np.int64), np.array(typ, np.int32), np.array(pos, np.float64),
            np.array(vel, np.float64), np.array(box, np.float64))


def read_lammps(path):
    with open(path) as f:
        lines = f.read().splitlines()
    it = iter(lines)
    line = next(it)
    while "atoms" not in line:
        line = next(it)
    n_atoms = int(line.split()[0])
    n_bonds = int(next(it).split()[0])
    n_angles = int(next(it).split()[0])
    while "xlo" not in line:
        line = next(it)
    lo_hi = [tuple(map(float, line.split()[0:2]))]
    lo_hi.append(tuple(map(float, next(it).split()[0:2])))
    lo_hi.append(tuple(map(float, next(it).split()[0:2])))
    box = np.array([hi - lo for lo, hi in lo_hi], np.float64)
    while "Atoms" not in line:
        line = next(it)
    next(it)
    milli = np.empty((n_atoms, 3), np.int64)
    for i in range(n_atoms):
        t = next(it).split()
        for k in range(3):
            s = t[3 + k]
            v = float(s)
            m = int(round(v * 1000.0))
            assert m / 1000.0 == v, (s, m)
            milli[i, k] = m
    while "Bonds" not in line:
        line = next(it)
    next(it)
    bonds = np.empty((n_bonds, 2), np.int64)
    for i in range(n_bonds):
        t = next(it).split()
        bonds[i] = (int(t[2]), int(t[3]))
    while "Angles" not in line:
        line = next(it)
    next(it)
    angles = np.empty((n_angles, 3), np.int64)
    for i in range(n_angles):
        t = next(it).split()
        angles[i] = (int(t[2]), int(t[3]), int(t[4]))
    return milli, bonds, angles, box


def main(ref_root):
    pid, typ, pos, vel, box = read_xyz(
        os.path.join(ref_root, "testsuite/verlet_list_buffer/lennard_jones_fluid_10000.xyz"))
    np.savez_compressed(os.path.join(HERE, "lj_fluid_2048.npz"), pid=pid, type=typ, pos=pos,
                        vel=vel, box=box)

    milli, bonds, angles, box = read_lammps(
        os.path.join(ref_root, "testsuite/tabulated/polymer_melt.start"))
    np.savez_compressed(os.path.join(HERE, "polymer_melt_40k.npz"),
                        pos_milli=milli.astype(np.int32), bonds=bonds.astype(np.int32),
                        angles=angles.astype(np.int32), box=box)

    # result.dat line "    0   0.0000    4.08575  0.01663   792677.003 ..." (no tabulation)
    with open(os.path.join(ref_root, "testsuite/tabulated/result.dat")) as f:
        lines = f.read().splitlines()
    start = [i for i, l in enumerate(lines) if "without tabulated" in l][0]
    row = [l for l in lines[start:] if l.split() and l.split()[0] == "0"][0].split()
    golden = {
        "source": "testsuite/tabulated/result.dat (simulation without tabulated potentials)",
        "step": 0, "T": float(row[1]), "P": float(row[2]), "Pxy": float(row[3]),
        "etotal": float(row[4]), "ekinetic": float(row[5]), "epair": float(row[6]),
        "ebond": float(row[7]), "eangle": float(row[8]),
        "setup": {"lj": {"epsilon": 1.0, "sigma": 1.0, "cutoff": 1.12, "shift": 0.0},
                  "fene": {"K": 30.0, "r0": 0.0, "rMax": 1.5},
                  "verlet_cutoff": 1.42, "skin": 0.3, "cell_grid": "decomp.cellGrid(rc=1.12)"},
        "printed_decimals": {"epair": 3, "ebond": 3, "P": 5},
    }
    # the same configuration with Tabulated(itype=2) tables written by the test script
    # (testsuite/tabulated/polymer_melt_tabulated.py writeTabFile: "%15.8g" x 3, N=257;
    # LJ r in [0.01, 1.12], FENE r in [0.0001, 1.49])
    start = [i for i, l in enumerate(lines) if "with tabulated" in l and "without" not in l][0]
    row = [l for l in lines[start:] if l.split() and l.split()[0] == "0"][0].split()
    golden["tabulated"] = {
        "source": "testsuite/tabulated/result.dat (simulation with tabulated potentials)",
        "P": float(row[2]), "Pxy": float(row[3]), "epair": float(row[6]),
        "ebond": float(row[7]),
        "tables": {"itype": 2, "N": 257, "format": "%15.8g %15.8g %15.8g\\n",
                   "lj": [0.01, 1.12], "fene": [0.0001, 1.49]},
    }
    with open(os.path.join(HERE, "polymer_melt_40k.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ESPRESSOPP_SRC")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set ESPRESSOPP_SRC)")
    main(root)
