"""tools.velocities.gaussian (src/tools/velocities.py:27-95)."""
import random


def gaussian(T, N, particle_mass=None, zero_momentum=True, seed=7654321, kb=1.0):
    random.seed(seed)
    bf = kb * T
    ekin = 0.0
    vx, vy, vz = [], [], []
    for i in range(N):
        mass = particle_mass[i] if particle_mass else 1.0
        sd = (bf / mass) ** 0.5
        for out in (vx, vy, vz):
            v = sd * random.gauss(0.0, 1.0)
            ekin += 0.5 * mass * v * v
            out.append(v)
    local_temp = (2.0 * ekin) / (3 * N * kb)
    if local_temp > 0:
        s = (T / local_temp) ** 0.5
        vx = [v * s for v in vx]
        vy = [v * s for v in vy]
        vz = [v * s for v in vz]
    if zero_momentum:
        mx, my, mz = sum(vx) / N, sum(vy) / N, sum(vz) / N
        vx = [v - mx for v in vx]
        vy = [v - my for v in vy]
        vz = [v - mz for v in vz]
    return vx, vy, vz
