"""tools.replicate (src/tools/replicate.py): a configuration with bonds and angles copied
xdim x ydim x zdim times along the box edges."""


def replicate(bonds, angles, x, y, z, Lx, Ly, Lz, xdim=1, ydim=1, zdim=1):
    """Returns (bonds, angles, x, y, z, Lx, Ly, Lz) of the replicated system.  Copies are
    appended in (i, j, k) loop order with k fastest, the original first; the c-th copy
    shifts positions by (i Lx, j Ly, k Lz) and particle ids in bonds and angles by
    c times the original particle count."""
    n = len(x)
    xs, ys, zs = list(x), list(y), list(z)
    bs, an = list(bonds), list(angles)
    copy = 0
    for i in range(xdim):
        for j in range(ydim):
            for k in range(zdim):
                if i + j + k == 0:
                    continue
                copy += 1
                xs.extend(v + i * Lx for v in x)
                ys.extend(v + j * Ly for v in y)
                zs.extend(v + k * Lz for v in z)
                off = copy * n
                bs.extend((p1 + off, p2 + off) for p1, p2 in bonds)
                an.extend((p1 + off, p2 + off, p3 + off) for p1, p2, p3 in angles)
    return bs, an, xs, ys, zs, xdim * Lx, ydim * Ly, zdim * Lz
