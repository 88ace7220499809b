"""verb4d_b200: the VERB-4D operator-split Fokker-Planck step on B200 (sm_100a).

Modules:
  _lib      ctypes binding of the C ABI (include/verb4d_b200.h)
  ops       per-slice operators with the reference's Python operator interface
  solver    device-resident Context and the whole-step Solver
  workload  seeded synthetic inputs of the benchmark configurations
"""
from . import _lib, ops, solver, workload  # noqa: F401
from ._lib import VerbError, load  # noqa: F401
from .ops import (BoundaryConditionType, Convection_1D, Convection_2D, Diffusion_1D,  # noqa: F401
                  Diffusion_2D, tridag)
from .solver import Context, Solver  # noqa: F401

__all__ = ["Context", "Solver", "VerbError", "load", "ops", "solver", "workload",
           "BoundaryConditionType", "Convection_1D", "Convection_2D", "Diffusion_1D",
           "Diffusion_2D", "tridag"]
