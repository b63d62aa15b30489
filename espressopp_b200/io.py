"""io.DumpXYZ (src/io/DumpXYZ.py:114-135, DumpXYZ.hpp:45-150, DumpXYZ.cpp:43-106) and
the file backup it makes when it does not append (src/io/FileBackup.hpp:37-70).

A dump downloads the particle state from the GPU once and writes one xyz frame: the
particle count, a comment line with the box, the integrator step and the length unit,
and one line per particle in ascending id order: [id] type x y z [vx vy vz], coordinates
in fixed notation with 10 decimals and scaled by length_factor (the velocities too, as in
the reference)."""
import os
import time

import numpy as np

_MONTHS = ("Jan", "Feb", "Mar", "Apr", "May", "Jun", "Jul", "Aug", "Sep", "Oct", "Nov", "Dec")


def _backup(file_name):
    """Moves an existing file_name to <year><Mon><day>_<hour><minute>_<file_name>."""
    if not os.path.exists(file_name):
        return
    t = time.localtime()
    new_name = "%04d%s%02d_%02d%02d_%s" % (t.tm_year, _MONTHS[t.tm_mon - 1], t.tm_mday,
                                           t.tm_hour, t.tm_min, file_name)
    print("Note: file %s exists already. Moving %s to %s" % (file_name, file_name, new_name))
    if os.path.exists(new_name):
        raise RuntimeError("Warning: can not backup file %s to %s, because it exists already!"
                           % (file_name, new_name))
    os.rename(file_name, new_name)


def _g6(v):
    """A double as an output stream of default precision prints it (6 significant)."""
    return "%g" % v


class DumpXYZ:
    """io.DumpXYZ(system, integrator, filename='out.xyz', unfolded=False,
    length_factor=1.0, length_unit='LJ', store_pids=False, store_velocities=False,
    append=True)."""

    def __init__(self, system, integrator, filename="out.xyz", unfolded=False,
                 length_factor=1.0, length_unit="LJ", store_pids=False,
                 store_velocities=False, append=True):
        self.system = system
        self.integrator = integrator
        self.filename = str(filename)
        self.unfolded = bool(unfolded)
        self.length_factor = float(length_factor)
        self.length_unit = str(length_unit)
        self.store_pids = bool(store_pids)
        self.store_velocities = bool(store_velocities)
        self.append = bool(append)
        if not self.append:
            _backup(self.filename)

    def dump(self):
        st = self.system.storage
        if st is None:
            raise RuntimeError("system has no storage")
        ids, pos, vel, _, img = st.getAll()
        L = np.asarray(self.system.bc.boxL, np.float64)
        if self.unfolded:
            pos = pos + img * L
        lf = self.length_factor
        lines = [str(len(ids)),
                 "%s  0.0  0.0  0.0  %s  0.0  0.0  0.0  %s  currentStep %d  lengthUnit %s" % (
                     _g6(L[0] * lf), _g6(L[1] * lf), _g6(L[2] * lf), int(self.integrator.step),
                     self.length_unit)]
        for k, pid in enumerate(ids):
            head = "%d " % pid if self.store_pids else ""
            line = head + "%d %.10f %.10f %.10f" % (st._types[int(pid)], lf * pos[k, 0],
                                                     lf * pos[k, 1], lf * pos[k, 2])
            if self.store_velocities:
                line += " %.10f %.10f %.10f" % (lf * vel[k, 0], lf * vel[k, 1], lf * vel[k, 2])
            lines.append(line)
        with open(self.filename, "a") as f:
            f.write("\n".join(lines) + "\n")
