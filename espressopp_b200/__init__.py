"""B200-native drop-in for ESPResSo++'s short-range MD step.

    import espressopp_b200 as espressopp

gives the classes a script of the reference uses for that step: System,
storage.DomainDecomposition, bc.OrthorhombicBC, esutil.RNG, VerletList, FixedPairList,
interaction.LennardJones / LennardJonesCapped / FENE with VerletListLennardJones /
VerletListLennardJonesCapped / FixedPairListFENE, integrator.VelocityVerlet /
LangevinThermostat / CapForce, analysis.Temperature / Pressure / PressureTensor, tools
and standard_system.  Particles live on the GPU (libespp_b200.so, C ABI in
include/espp_b200.h); there is no CPU fallback.
"""
from ._lib import LIBRARY_PATH, load_library  # noqa: F401
from .core import (FixedPairList, FixedTripleList, Int3D, Real3D, System,  # noqa: F401
                   Tensor, VerletList, infinity, set_default_precision)
from . import analysis, bc, esutil, integrator, interaction, io, storage, tools  # noqa: F401
from . import standard_system  # noqa: F401
from .parallel_tempering import ParallelTempering  # noqa: F401
from ._mpi import MPI  # noqa: F401

__all__ = ["System", "VerletList", "FixedPairList", "FixedTripleList", "Real3D", "Int3D",
           "Tensor", "analysis",
           "bc", "esutil", "integrator", "interaction", "storage", "tools", "standard_system",
           "set_default_precision", "load_library", "infinity", "ParallelTempering", "MPI"]
