"""Solvers (``newton.solvers``): the B200 VBD particle solver."""

from .solver import SolverBase
from .solver_vbd import SolverVBD

__all__ = ["SolverBase", "SolverVBD"]
