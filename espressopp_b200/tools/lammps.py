"""tools.lammps.read (src/tools/lammps.py:33-120): atoms, bonds and angles."""


def read(fin):
    with open(fin) as f:
        line = f.readline()
        while "atoms" not in line:
            line = f.readline()
        num_particles = int(line.split()[0])
        num_bonds = int(f.readline().split()[0])
        num_angles = int(f.readline().split()[0])
        while "xlo" not in line:
            line = f.readline()
        xmin, xmax = map(float, line.split()[0:2])
        ymin, ymax = map(float, f.readline().split()[0:2])
        zmin, zmax = map(float, f.readline().split()[0:2])
        while "Atoms" not in line:
            line = f.readline()
        f.readline()
        x, y, z = [], [], []
        for _ in range(num_particles):
            t = f.readline().split()
            x.append(float(t[-3]))
            y.append(float(t[-2]))
            z.append(float(t[-1]))
        bonds, angles = [], []
        if num_bonds:
            while "Bonds" not in line:
                line = f.readline()
            f.readline()
            for _ in range(num_bonds):
                t = f.readline().split()
                bonds.append((int(t[2]), int(t[3])))
        if num_angles:
            while "Angles" not in line:
                line = f.readline()
            f.readline()
            for _ in range(num_angles):
                t = f.readline().split()
                angles.append((int(t[2]), int(t[3]), int(t[4])))
    return bonds, angles, x, y, z, xmax - xmin, ymax - ymin, zmax - zmin
