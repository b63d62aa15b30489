"""tools.lammps.read (src/tools/lammps.py:33-155): a LAMMPS data file's atoms, bonds,
angles, dihedrals and velocities, returned in the reference's shapes."""


def _skip_to(f, word):
    line = ""
    while word not in line:
        line = f.readline()
        if line == "":
            raise ValueError("LAMMPS data file has no '%s' section" % word)
    return line


def _rows(f, n, first, conv):
    out = []
    for _ in range(n):
        out.append([conv(v) for v in f.readline().split()[first:]])
    return out


def read(fin):
    """Header: the counts of atoms, bonds, angles and dihedrals on consecutive lines, then
    the impropers line, a blank line and the atom-types line (which may carry the word
    'velocities'); then the box, and the Atoms / Bonds / Angles / Dihedrals / Velocities
    sections.  With one atom type an atom line ends with x y z (the coordinates start at
    column 3, or 2 when there are no bonds); with several it is id mol type q x y z.

    Returns, as the reference does:
      several atom types:        p_type, bonds, angles, q, x, y, z, Lx, Ly, Lz
      atoms only:                x, y, z, Lx, Ly, Lz (+ vx, vy, vz with 'velocities')
      bonds:                     bonds, x, y, z, Lx, Ly, Lz
      bonds and angles:          bonds, angles, x, y, z, Lx, Ly, Lz
      otherwise:                 bonds, angles, dihedrals, x, y, z, Lx, Ly, Lz
    """
    with open(fin) as f:
        line = _skip_to(f, "atoms")
        num_particles = int(line.split()[0])
        num_bonds = int(f.readline().split()[0])
        num_angles = int(f.readline().split()[0])
        num_dihedrals = int(f.readline().split()[0])
        f.readline()  # impropers
        f.readline()  # blank line
        line = f.readline()
        num_types = int(line.split()[0])
        velocities = "velocities" in line

        line = _skip_to(f, "xlo")
        xmin, xmax = map(float, line.split()[0:2])
        ymin, ymax = map(float, f.readline().split()[0:2])
        zmin, zmax = map(float, f.readline().split()[0:2])
        Lx, Ly, Lz = xmax - xmin, ymax - ymin, zmax - zmin

        _skip_to(f, "Atoms")
        f.readline()
        x, y, z = [], [], []
        p_type, q = [], []
        if num_types == 1:
            first = 3 if num_bonds else 2
            for rx, ry, rz in _rows(f, num_particles, first, float):
                x.append(rx)
                y.append(ry)
                z.append(rz)
        else:
            for k, rq, rx, ry, rz in _rows(f, num_particles, 2, float):
                p_type.append(int(k))
                q.append(rq)
                x.append(rx)
                y.append(ry)
                z.append(rz)

        bonds = angles = dihedrals = None
        if num_bonds:
            _skip_to(f, "Bonds")
            f.readline()
            bonds = [(r[0], r[1]) for r in _rows(f, num_bonds, 2, int)]
        if num_angles:
            _skip_to(f, "Angles")
            f.readline()
            angles = [tuple(r) for r in _rows(f, num_angles, 2, int)]
        if num_dihedrals:
            _skip_to(f, "Dihedrals")
            f.readline()
            dihedrals = [tuple(r) for r in _rows(f, num_dihedrals, 2, int)]
        if velocities:
            _skip_to(f, "Velocities")
            f.readline()
            v = _rows(f, num_particles, 1, float)
            vx = [r[0] for r in v]
            vy = [r[1] for r in v]
            vz = [r[2] for r in v]

    if num_types != 1:
        return p_type, bonds, angles, q, x, y, z, Lx, Ly, Lz
    if not num_bonds and not num_angles and not num_dihedrals:
        if velocities:
            return x, y, z, Lx, Ly, Lz, vx, vy, vz
        return x, y, z, Lx, Ly, Lz
    if num_bonds and not num_angles and not num_dihedrals:
        return bonds, x, y, z, Lx, Ly, Lz
    if num_bonds and num_angles and not num_dihedrals:
        return bonds, angles, x, y, z, Lx, Ly, Lz
    return bonds, angles, dihedrals, x, y, z, Lx, Ly, Lz
