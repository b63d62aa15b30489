"""Setup and reporting helpers mirroring espressopp.tools.  As in the reference package,
the helper functions are also reachable at package level (tools.info, tools.readxyz,
tools.replicate, ...)."""
from . import analyse, decomp, lammps, lattice, timers, topology, velocities  # noqa: F401
from .analyse import *  # noqa: F401,F403
from .decomp import *  # noqa: F401,F403
from .DumpConfigurations import *  # noqa: F401,F403
from .lattice import *  # noqa: F401,F403
from .replicate import replicate  # noqa: F401
