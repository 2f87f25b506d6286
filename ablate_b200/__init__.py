"""B200-native backend for ABLATE's finite-volume right-hand side (FiniteVolumeSolver::ComputeRHSFunction).

The compute path is the sm_100a CUDA library ``lib/libablate_fv.so`` behind the C ABI of
``include/ablate_fv.h``; this package is its host-side binding and the mirror of the reference's
process/EOS/flux-calculator interfaces (``fv``) plus synthetic mesh builders (``mesh``).
"""
from . import _lib
from .fv import (Ausm, AusmpUp, AverageFlux, Constant, ConstantLewis, FiniteVolumeSolver, NavierStokesTransport, OffFlux,
                 PerfectGas, PressureGradientScaling, Riemann, SpeciesTransport, Sutherland, TChem, eos_property, make_physics)
from .mesh import Mesh, box_mesh

__all__ = ["Ausm", "AusmpUp", "AverageFlux", "Constant", "ConstantLewis", "FiniteVolumeSolver", "NavierStokesTransport", "OffFlux",
           "PerfectGas", "PressureGradientScaling", "Riemann", "SpeciesTransport", "Sutherland", "TChem", "eos_property",
           "make_physics", "Mesh", "box_mesh"]
