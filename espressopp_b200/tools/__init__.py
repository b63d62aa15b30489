"""Setup and reporting helpers mirroring espressopp.tools."""
from . import analyse, decomp, lammps, lattice, timers, topology, velocities  # noqa: F401
from .DumpConfigurations import readxyz, writexyz  # noqa: F401
