"""Solvers: SolverBase (integrate_particles), the WCSPH SolverSPH and its
differentiable step / checkpointed rollout (sph_diff)."""

from .flags import SolverNotifyFlags
from .solver import SolverBase
from .sph import SPHConfig, SolverSPH
from .sph_diff import checkpoint_schedule, sph_rollout, sph_step

__all__ = ["SPHConfig", "SolverBase", "SolverNotifyFlags", "SolverSPH", "checkpoint_schedule", "sph_rollout",
           "sph_step"]
