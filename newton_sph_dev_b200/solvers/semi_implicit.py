"""SolverSemiImplicit for particles, mirroring the particle path of
newton/_src/solvers/semi_implicit/solver_semi_implicit.py (step :95-185):
particle-particle contact forces on the HashGrid (written into
state_in.particle_f for active particles, as eval_particle_contact does),
then the particle-shape contact forces of the soft contacts subtracted from
it, then integrate_particles. As in the reference, the solver does not build
the grid: the caller builds ``model.particle_grid`` on state_in's positions
(with cell width 2 * particle_max_radius + particle_cohesion) when particle
contacts are wanted; an unbuilt grid means no particle-particle forces.

Rigid bodies, springs, triangles, tetrahedra and joints are not part of this
library's particle path: a model that has them is refused.
"""

from __future__ import annotations

from .. import contacts as pc
from ..sim import Control, Model, State
from .solver import SolverBase


class SolverSemiImplicit(SolverBase):
    """Semi-implicit Euler for particles with penalty contacts."""

    def __init__(self, model: Model, angular_damping: float = 0.05, friction_smoothing: float = 1.0,
                 joint_attach_ke: float = 1.0e4, joint_attach_kd: float = 1.0e2, enable_tri_contact: bool = True):
        super().__init__(model)
        for name in ("body_count", "joint_count", "tri_count", "tet_count"):
            if getattr(model, name, 0):
                raise NotImplementedError(f"SolverSemiImplicit here simulates particles only (model.{name} > 0)")
        self.angular_damping = angular_damping
        self.friction_smoothing = friction_smoothing
        self.joint_attach_ke = joint_attach_ke
        self.joint_attach_kd = joint_attach_kd
        self.enable_tri_contact = enable_tri_contact

    def step(self, state_in: State, state_out: State, control: Control | None, contacts, dt: float) -> None:
        model = self.model
        if not state_in.particle_count:
            return
        particle_f = state_in.particle_f
        pc.eval_particle_contact_forces(model, state_in, particle_f)
        pc.eval_particle_body_contact_forces(model, state_in, contacts, particle_f)
        self.integrate_particles(model, state_in, state_out, dt)


__all__ = ["SolverSemiImplicit"]
