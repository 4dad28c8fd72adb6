"""SolverBase, mirroring newton/_src/solvers/solver.py:177-366 for particles.

``integrate_particles`` launches the sm_100a kernel behind
``nsph_integrate_particles`` (replacing the Warp kernel at solver.py:10-47).
"""

from __future__ import annotations

import torch

from .. import _lib
from ..sim import Control, Model, ModelBuilder, State


def _require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise RuntimeError(f"{name} is on {t.device}: the solvers run on CUDA only (there is no CPU fallback)")


class SolverBase:
    """Generic solver base class (solver.py:177)."""

    def __init__(self, model: Model):
        self.model = model

    @property
    def device(self) -> torch.device:
        """Device of the model the solver runs on."""
        return self.model.device

    def integrate_particles(self, model: Model, state_in: State, state_out: State, dt: float) -> None:
        """Symplectic Euler for particles (solver.py:266-299, kernel :10-47):
        ``v1 = v0 + (f*w + g*step(-w))*dt``, ``|v1|`` clamped to
        ``model.particle_max_velocity``, ``x1 = x0 + v1*dt``; inactive
        particles copy x and leave ``state_out.particle_qd`` untouched."""
        if not model.particle_count:
            return
        _require_cuda(state_in.particle_q, "state_in.particle_q")
        lib = _lib.load()
        st = lib.nsph_integrate_particles(
            state_in.particle_q.data_ptr(),
            state_in.particle_qd.data_ptr(),
            state_in.particle_f.data_ptr(),
            model.particle_inv_mass.data_ptr(),
            model.particle_flags.data_ptr(),
            model.particle_world.data_ptr(),
            model.gravity.data_ptr(),
            int(model.gravity.shape[0]),
            int(model.particle_count),
            float(dt),
            float(model.particle_max_velocity),
            state_out.particle_q.data_ptr(),
            state_out.particle_qd.data_ptr(),
            _lib.stream_handle(model.device),
        )
        _lib.check(st, "integrate_particles")

    def step(self, state_in: State, state_out: State, control: Control | None, contacts, dt: float) -> None:
        """Advance the model by dt from state_in to state_out."""
        raise NotImplementedError()

    def notify_model_changed(self, flags: int) -> None:
        """Tell the solver which model properties changed (solver.py:318-345)."""

    def update_contacts(self, contacts, state: State | None = None) -> None:
        raise NotImplementedError()

    @classmethod
    def register_custom_attributes(cls, builder: ModelBuilder) -> None:
        """Register solver-specific custom attributes on a builder (solver.py:358-366)."""


__all__ = ["SolverBase"]
