"""Solvers: SolverBase (integrate_particles) and the WCSPH SolverSPH."""

from .flags import SolverNotifyFlags
from .solver import SolverBase
from .sph import SPHConfig, SolverSPH

__all__ = ["SPHConfig", "SolverBase", "SolverNotifyFlags", "SolverSPH"]
