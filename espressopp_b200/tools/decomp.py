"""tools.decomp (src/tools/decomp.py:100-342) for one node."""
from ..core import Int3D


def nodeGrid(n=1, box_size=None, rc=None, skin=None, eh_size=0, ratioMS=0, idealGas=0,
             slabMSDims=None):
    """The node grid for n nodes (tools/decomp.py:28-320).  The GPU storage decomposes
    space into slabs along z, so n nodes give (1, 1, n); the reference's balanced 3-d
    factorisation is not used."""
    n = int(n)
    if n < 1:
        raise ValueError("the number of nodes must be positive")
    return Int3D(1, 1, n)


def nodeGridSimple(n=1):
    return nodeGrid(n)


def cellGrid(box_size, node_grid, rc, skin, halfCellInt=1):
    rc_skin = rc + skin
    if rc_skin == 0:
        raise ValueError("interaction range (cutoff + skin) must be larger than 0")
    if node_grid[0] <= 0 or node_grid[1] <= 0 or node_grid[2] <= 0:
        raise ValueError("invalid node grid %s" % str(node_grid))
    out = []
    for k in range(3):
        v = (box_size[k] * halfCellInt) / (rc_skin * node_grid[k])
        if v < 1:
            raise ValueError("local box size in direction %d (=%6f) is smaller than interaction "
                             "range (cutoff + skin = %6f)" % (k, v, rc_skin))
        out.append(int(v))
    return Int3D(out)
