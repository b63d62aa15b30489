"""tools.lattice.createCubic (src/tools/lattice.py:24-71)."""
import random


def createCubic(N, rho, perfect=True, RNG=None):
    L = (N / rho) ** (1.0 / 3.0)
    a = int(N ** (1.0 / 3.0))
    if a ** 3 < N:
        a = a + 1
    spacing = L / a

    def rnd(m):
        u = random.random() if RNG is None else RNG()
        return m * (2.0 * u - 1.0)

    magn = 0.0 if perfect else spacing / 10.0
    x, y, z = [], [], []
    ct = 0
    for i in range(a):
        for j in range(a):
            for k in range(a):
                if ct < N:
                    x.append(0.5 * spacing + i * spacing + rnd(magn))
                    y.append(0.5 * spacing + j * spacing + rnd(magn))
                    z.append(0.5 * spacing + k * spacing + rnd(magn))
                    ct += 1
    return x, y, z, L, L, L
