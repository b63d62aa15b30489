"""readxyz / writexyz (src/tools/DumpConfigurations.py:60-145)."""


def readxyz(filename):
    with open(filename) as f:
        n = int(f.readline().split()[0])
        t = f.readline().split()
        if len(t) == 3:
            Lx, Ly, Lz = float(t[0]), float(t[1]), float(t[2])
        else:
            Lx, Ly, Lz = float(t[0]), float(t[4]), float(t[8])
        pid, typ, xp, yp, zp, xv, yv, zv = [], [], [], [], [], [], [], []
        for _ in range(n):
            t = f.readline().split()
            if len(t) in (7, 4):
                t.insert(1, "0")
            pid.append(int(t[0]))
            typ.append(int(t[1]))
            xp.append(float(t[2]))
            yp.append(float(t[3]))
            zp.append(float(t[4]))
            if len(t) > 5:
                xv.append(float(t[5]))
                yv.append(float(t[6]))
                zv.append(float(t[7]))
            else:
                xv.append(0.0)
                yv.append(0.0)
                zv.append(0.0)
    return pid, typ, xp, yp, zp, xv, yv, zv, Lx, Ly, Lz


def writexyz(filename, system, velocities=True, unfolded=False):
    st = system.storage
    ids, pos, vel, _, img = st.getAll()
    L = system.bc.boxL
    with open(filename, "w") as f:
        f.write("%d\n" % len(ids))
        f.write("%15.10f %15.10f %15.10f\n" % (L[0], L[1], L[2]))
        for k, pid in enumerate(ids):
            p = pos[k] + (img[k] * L if unfolded else 0.0)
            line = "%d %d %15.10f %15.10f %15.10f" % (pid, st._types[int(pid)], p[0], p[1], p[2])
            if velocities:
                line += " %15.10f %15.10f %15.10f" % tuple(vel[k])
            f.write(line + "\n")
