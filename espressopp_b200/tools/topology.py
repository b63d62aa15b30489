"""Polymer set-up helpers (espressopp.tools.topology).

``polymerRW`` mirrors the reference's random-walk chain generator
(src/tools/topology.py:27-130).  ``polymer_melt`` builds a Kremer-Grest melt: chains
grown as random walks from random starting points in a periodic cubic box, each new bead
placed at the bond length from the previous one in a direction drawn uniformly on the
sphere and rejected while it comes closer than ``mindist`` to any bead already placed
(neighbour search on a cell grid).  A bead that finds no free direction in ``tries``
draws takes the best direction seen; the short-range overlaps this leaves are what the
force-capped warm-up of a Kremer-Grest run removes.
"""
import math
import random

import numpy as np

from ..core import Real3D


def polymerRW(pid, startpos, numberOfMonomers, bondlength, return_angles=False,
              return_dihedrals=False, mindist=None, rng=None):
    """Random-walk chain of numberOfMonomers beads starting at startpos; with mindist the
    bead after next must lie farther than mindist from the previous one
    (tools/topology.py:27-130).  Returns positions, bonds[, angles][, dihedrals]
    [, average cos(theta)] as the reference does."""
    draw = rng if rng is not None else (lambda: random.uniform(0, 1))
    x, y, z = startpos[0], startpos[1], startpos[2]
    positions = [Real3D(x, y, z)]
    bonds, angles, dihedrals = [], [], []
    avecostheta = 0.0
    for i in range(numberOfMonomers - 1):
        while True:
            nextZ = (2.0 * draw() - 1.0) * bondlength
            phi = 2.0 * math.pi * draw()
            rr = math.sqrt(bondlength * bondlength - nextZ * nextZ)
            nextX = rr * math.cos(phi)
            nextY = rr * math.sin(phi)
            if not (mindist and i > 0):
                break
            ax = positions[i][0] - positions[i - 1][0]
            ay = positions[i][1] - positions[i - 1][1]
            az = positions[i][2] - positions[i - 1][2]
            la = math.sqrt(ax * ax + ay * ay + az * az)
            bx, by, bz = -nextX, -nextY, -nextZ
            lb = math.sqrt(bx * bx + by * by + bz * bz)
            cx, cy, cz = ax - bx, ay - by, az - bz
            if math.sqrt(cx * cx + cy * cy + cz * cz) > mindist:
                avecostheta += -(ax * bx + ay * by + az * bz) / (la * lb)
                break
        x += nextX
        y += nextY
        z += nextZ
        positions.append(Real3D(x, y, z))
        bonds.append((pid + i, pid + i + 1))
        if return_angles and i < numberOfMonomers - 2:
            angles.append((pid + i, pid + i + 1, pid + i + 2))
        if return_dihedrals and i < numberOfMonomers - 3:
            dihedrals.append((pid + i, pid + i + 1, pid + i + 2, pid + i + 3))
    out = [positions, bonds]
    if return_angles:
        out.append(angles)
    if return_dihedrals:
        out.append(dihedrals)
    if mindist:
        out.append(avecostheta / max(numberOfMonomers - 2, 1))
    return tuple(out)


def polymer_melt(nchains, nbeads, density, bondlen=0.97, mindist=0.8, seed=3, tries=64):
    """Kremer-Grest melt of nchains x nbeads beads at bead density `density` in a cubic
    periodic box.  Returns (positions (N, 3), unwrapped along each chain so that bonded
    beads are one bond length apart, bonds (M, 2) of 1-based ids numbered chain by chain,
    box length L).  Seeded: numpy PCG64(seed)."""
    N = nchains * nbeads
    L = (N / density) ** (1.0 / 3.0)
    rng = np.random.Generator(np.random.PCG64(seed))
    # cells at least bond length + mindist wide: the 27 cells around a bead hold every
    # bead that can come within mindist of a candidate placed from it
    ncell = max(3, int(L / (bondlen + mindist)))
    csz = L / ncell
    grid = {}
    pos = np.empty((N, 3))    # wrapped into the box, for the neighbour search
    unw = np.empty((N, 3))    # unwrapped along the chains
    md2 = mindist * mindist

    def cell_of(p):
        return (math.floor(p[0] / csz) % ncell, math.floor(p[1] / csz) % ncell,
                math.floor(p[2] / csz) % ncell)

    def near(p):
        cx, cy, cz = cell_of(p)
        idx = []
        for ox in (-1, 0, 1):
            for oy in (-1, 0, 1):
                for oz in (-1, 0, 1):
                    lst = grid.get(((cx + ox) % ncell, (cy + oy) % ncell, (cz + oz) % ncell))
                    if lst:
                        idx.extend(lst)
        return pos[idx]

    def min_dist2(cands, nb):
        # squared distance of each candidate to its nearest placed bead (minimum image)
        if len(nb) == 0:
            return np.full(len(cands), np.inf)
        d = nb[None, :, :] - cands[:, None, :]
        d -= L * np.round(d / L)
        return np.min(np.einsum("ijk,ijk->ij", d, d), axis=1)

    def place(k, p):
        unw[k] = p
        p = p - L * np.floor(p / L)
        pos[k] = p
        grid.setdefault(cell_of(p), []).append(k)

    k = 0
    for _ in range(nchains):
        for _ in range(tries):
            start = rng.uniform(0.0, L, 3)
            if min_dist2(start[None, :], near(start))[0] >= md2:
                break
        place(k, start)
        k += 1
        for _ in range(nbeads - 1):
            prev = unw[k - 1].copy()
            nb = near(prev)
            best_c, best_d = None, -1.0
            for _ in range(0, tries, 8):
                z = rng.uniform(-1.0, 1.0, 8)
                phi = rng.uniform(0.0, 2.0 * math.pi, 8)
                rr = np.sqrt(1.0 - z * z)
                cands = prev + np.stack([rr * np.cos(phi), rr * np.sin(phi), z], 1) * bondlen
                dd = min_dist2(cands, nb)
                j = int(np.argmax(dd))
                if dd[j] > best_d:
                    best_c, best_d = cands[j], dd[j]
                if best_d >= md2:
                    break
            place(k, best_c)
            k += 1
    ids = np.arange(1, N + 1).reshape(nchains, nbeads)
    bonds = np.stack([ids[:, :-1].reshape(-1), ids[:, 1:].reshape(-1)], 1)
    return unw, bonds.astype(np.int64), L
