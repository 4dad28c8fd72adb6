"""Solvers: SolverBase (integrate_particles), the WCSPH SolverSPH and its
differentiable step / checkpointed rollout (sph_diff), and the particle
paths of SolverXPBD and SolverSemiImplicit."""

from .flags import SolverNotifyFlags
from .semi_implicit import SolverSemiImplicit
from .solver import SolverBase
from .sph import SPHConfig, SolverSPH
from .sph_diff import checkpoint_schedule, sph_rollout, sph_step
from .xpbd import SolverXPBD

__all__ = ["SPHConfig", "SolverBase", "SolverNotifyFlags", "SolverSPH", "SolverSemiImplicit", "SolverXPBD",
           "checkpoint_schedule", "sph_rollout", "sph_step"]
