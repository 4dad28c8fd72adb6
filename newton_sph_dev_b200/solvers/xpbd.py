"""SolverXPBD for particles, mirroring the particle path of
newton/_src/solvers/xpbd/solver_xpbd.py (SolverXPBD.__init__ :97-139,
_apply_particle_deltas :157-197, step :260-714):

1. integrate_particles from state_in into state_out (the prediction);
2. the HashGrid built on the predicted positions with cell width
   2 * particle_max_radius + particle_cohesion;
3. per iteration: zero the deltas, add the particle-shape corrections of the
   soft contacts (static shapes) and the particle-particle corrections, then
   apply_particle_deltas: x = x_pred + delta, v = (x - x_0)/dt, |v| clamped;
   iterates ping-pong between the two states' buffers as in the reference
   (so state_in's particle_q / particle_qd are overwritten by the step);
4. the final iterate in state_out, then, with enable_restitution, the
   restitution of approaching shape contacts.

Rigid bodies, springs, triangles, tetrahedra and joints are not part of this
library's particle path: a model that has them is refused.
"""

from __future__ import annotations

import torch

from .. import contacts as pc
from ..sim import Control, Model, State
from .solver import SolverBase, _require_cuda


class SolverXPBD(SolverBase):
    """Position-based particle solver (particle-particle and particle-shape
    contacts) on this library's kernels."""

    def __init__(self, model: Model, iterations: int = 2, soft_body_relaxation: float = 0.9,
                 soft_contact_relaxation: float = 0.9, joint_linear_relaxation: float = 0.7,
                 joint_angular_relaxation: float = 0.4, joint_linear_compliance: float = 0.0,
                 joint_angular_compliance: float = 0.0, rigid_contact_relaxation: float = 0.8,
                 rigid_contact_con_weighting: bool = True, angular_damping: float = 0.0,
                 enable_restitution: bool = False):
        super().__init__(model)
        for name in ("body_count", "joint_count", "tri_count", "tet_count"):
            if getattr(model, name, 0):
                raise NotImplementedError(f"SolverXPBD here simulates particles only (model.{name} > 0)")
        self.iterations = int(iterations)
        self.soft_body_relaxation = soft_body_relaxation
        self.soft_contact_relaxation = soft_contact_relaxation
        self.enable_restitution = enable_restitution
        self._particle_delta_counter = 0
        self._deltas = None
        self._q_init = None
        self._qd_init = None
        if model.particle_count:
            _require_cuda(model.particle_q, "model.particle_q")
            self._deltas = torch.empty_like(model.particle_q)
            self._q_init = torch.empty_like(model.particle_q)
            self._qd_init = torch.empty_like(model.particle_q)
        if model.particle_count > 1 and model.particle_grid is not None:
            model.particle_grid.reserve(model.particle_count)

    def _apply_particle_deltas(self, model: Model, state_in: State, state_out: State, dt: float):
        """One apply_particle_deltas, alternating the buffers as the reference does."""
        if self._particle_delta_counter == 0:
            particle_q = state_out.particle_q
            new_q, new_qd = state_in.particle_q, state_in.particle_qd
        else:
            particle_q = state_in.particle_q
            new_q, new_qd = state_out.particle_q, state_out.particle_qd
        self._particle_delta_counter = 1 - self._particle_delta_counter
        pc.apply_particle_deltas(model, self._q_init, particle_q, self._deltas, dt, new_q, new_qd)
        return new_q, new_qd

    def step(self, state_in: State, state_out: State, control: Control | None, contacts, dt: float) -> None:
        model = self.model
        if state_in.requires_grad:
            raise NotImplementedError("SolverXPBD here has no gradient path")
        self._particle_delta_counter = 0
        if not model.particle_count:
            return
        particle_q, particle_qd = state_out.particle_q, state_out.particle_qd
        self._q_init.copy_(state_in.particle_q)
        if self.enable_restitution:
            self._qd_init.copy_(state_in.particle_qd)
        self.integrate_particles(model, state_in, state_out, dt)
        if model.particle_count > 1 and model.particle_grid is not None:
            search_radius = model.particle_max_radius * 2.0 + model.particle_cohesion
            model.particle_grid.build(state_out.particle_q, radius=search_radius)
        for _ in range(self.iterations):
            self._deltas.zero_()
            if model.shape_count:
                pc.solve_particle_shape_contacts(model, particle_q, particle_qd, contacts, self._deltas, dt,
                                                 self.soft_contact_relaxation)
            if model.particle_max_radius > 0.0 and model.particle_count > 1:
                pc.solve_particle_particle_contacts(model, particle_q, particle_qd, self._deltas, dt,
                                                    self.soft_contact_relaxation)
            particle_q, particle_qd = self._apply_particle_deltas(model, state_in, state_out, dt)
        if particle_q.data_ptr() != state_out.particle_q.data_ptr():
            state_out.particle_q.copy_(particle_q)
            state_out.particle_qd.copy_(particle_qd)
        if self.enable_restitution and contacts is not None:
            pc.apply_particle_shape_restitution(model, contacts, particle_qd, self._q_init, self._qd_init,
                                                state_out.particle_qd)


__all__ = ["SolverXPBD"]
