"""B200-native differentiable lattice-Boltzmann density-design solver.

The product is the CUDA library ``liblbm_b200.so`` (C-ABI in
include/lbm_b200.h); this package holds its build step and the Python mirror
of the reference provider interface.
"""
from .problem import ContractError, NormalizedProblem, SolverOptions, normalize
from .solver import RESPONSES, AdjointReport, ConvergenceError, CudaError, Diagnostics, LbmSolver, StateError

__all__ = [
    "ContractError",
    "ConvergenceError",
    "CudaError",
    "StateError",
    "NormalizedProblem",
    "SolverOptions",
    "normalize",
    "RESPONSES",
    "AdjointReport",
    "Diagnostics",
    "LbmSolver",
]
