"""Static particle model, mirroring the particle part of
newton/_src/sim/model.py (fields :140-178, gravity :631, particle_count :691,
state() :827-878, control() :880, set_gravity() :923-956).

Storage is torch tensors on the model's device (the reference uses
``wp.array``); vec3 arrays have shape ``(N, 3)`` float32.
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import IntEnum
from typing import Any

import numpy as np
import torch

from .control import Control
from .state import AttributeNamespace, State


class Model:
    """Particle model: per-particle static data, gravity and the hash grid."""

    class AttributeFrequency(IntEnum):
        """How many values a custom attribute holds (model.py:65-91)."""

        ONCE = 0
        PARTICLE = 4

    class AttributeAssignment(IntEnum):
        """Which object a custom attribute is attached to."""

        MODEL = 0
        STATE = 1
        CONTROL = 2

    @dataclass
    class CustomAttributeSpec:
        name: str
        namespace: str | None
        frequency: int
        assignment: int
        dtype: torch.dtype
        width: int
        default: Any

    def __init__(self, device: str | torch.device = "cuda:0"):
        self.device = torch.device(device)
        self.requires_grad: bool = False
        self.world_count: int = 0
        self.up_axis: int = 2

        self.particle_q: torch.Tensor | None = None
        """Particle positions [m], shape (particle_count, 3), float32."""
        self.particle_qd: torch.Tensor | None = None
        """Particle velocities [m/s], shape (particle_count, 3), float32."""
        self.particle_mass: torch.Tensor | None = None
        """Particle mass [kg], shape (particle_count,), float32."""
        self.particle_inv_mass: torch.Tensor | None = None
        """Particle inverse mass [1/kg] (0 for zero mass), float32."""
        self.particle_radius: torch.Tensor | None = None
        """Particle radius [m], float32."""
        self.particle_flags: torch.Tensor | None = None
        """Particle flags (ParticleFlags bits), int32."""
        self.particle_world: torch.Tensor | None = None
        """World index per particle, int32; -1 for global particles."""
        self.particle_world_start: torch.Tensor | None = None
        self.particle_max_radius: float = 0.0
        self.particle_max_velocity: float = 1e5
        """Maximum particle speed [m/s] (velocity clamp)."""
        self.particle_ke: float = 1.0e3
        self.particle_kd: float = 1.0e2
        self.particle_kf: float = 1.0e2
        self.particle_mu: float = 0.5
        self.particle_cohesion: float = 0.0
        self.particle_adhesion: float = 0.0
        self.particle_grid = None
        """HashGrid for particle interactions (HashGrid(128,128,128) when the
        model has more than one particle of positive radius on a CUDA device)."""
        self.gravity: torch.Tensor | None = None
        """Per-world gravity [m/s^2], shape (world_count, 3), float32. Solvers
        read it on the device at every step, so set_gravity takes effect
        without recapturing a CUDA graph."""
        self.particle_count: int = 0
        self.body_count: int = 0
        self.shape_count: int = 0
        self.joint_count: int = 0
        self.tri_count: int = 0
        self.tet_count: int = 0
        self.muscle_count: int = 0
        self.custom_attributes: dict[str, Model.CustomAttributeSpec] = {}
        self._requested_state_attributes: set[str] = set()

    # ------------------------------------------------------------------
    def state(self, requires_grad: bool | None = None) -> State:
        """New State initialised from the model: q and qd cloned, f zeroed,
        STATE-assigned custom attributes allocated (model.py:827-878)."""
        if requires_grad is None:
            requires_grad = self.requires_grad
        s = State()
        if self.particle_count:
            s.particle_q = self.particle_q.clone().requires_grad_(requires_grad)
            s.particle_qd = self.particle_qd.clone().requires_grad_(requires_grad)
            s.particle_f = torch.zeros_like(self.particle_qd).requires_grad_(requires_grad)
        self._add_custom_attributes(s, Model.AttributeAssignment.STATE)
        return s

    def control(self, requires_grad: bool | None = None, clone_variables: bool = True) -> Control:
        """New Control (model.py:880); empty for a particle-only model."""
        c = Control()
        self._add_custom_attributes(c, Model.AttributeAssignment.CONTROL)
        return c

    def set_gravity(self, gravity, world: int | None = None) -> None:
        """Set gravity at runtime (model.py:923-956).

        Args:
            gravity: a vector (3,) for every world, or an array (world_count, 3).
            world: when given, set only this world's gravity.

        Call ``solver.notify_model_changed(SolverNotifyFlags.MODEL_PROPERTIES)``
        afterwards; the new values are read on the device by the next step,
        also from a replayed CUDA graph.
        """
        g = np.asarray(gravity, dtype=np.float32)
        if world is not None:
            if g.shape != (3,):
                raise ValueError("Expected single gravity vector (3,) when world is specified")
            if world < 0 or world >= self.world_count:
                raise IndexError(f"world {world} out of range [0, {self.world_count})")
            self.gravity[world].copy_(torch.from_numpy(g))
        elif g.ndim == 1:
            self.gravity.copy_(torch.from_numpy(np.broadcast_to(g, (self.world_count, 3)).copy()))
        else:
            if len(g) != self.world_count:
                raise ValueError(f"Expected {self.world_count} gravity vectors, got {len(g)}")
            self.gravity.copy_(torch.from_numpy(g))

    def request_state_attributes(self, *names: str) -> None:
        self._requested_state_attributes.update(names)

    def get_requested_state_attributes(self) -> set[str]:
        return set(self._requested_state_attributes)

    # ------------------------------------------------------------------
    def _add_custom_attributes(self, target, assignment: int) -> None:
        for key, spec in self.custom_attributes.items():
            if spec.assignment != assignment:
                continue
            if spec.frequency == Model.AttributeFrequency.PARTICLE:
                shape = (self.particle_count,) if spec.width == 1 else (self.particle_count, spec.width)
            else:
                shape = (1,) if spec.width == 1 else (1, spec.width)
            t = torch.full(shape, spec.default, dtype=spec.dtype, device=self.device)
            holder = target
            if spec.namespace:
                holder = getattr(target, spec.namespace, None)
                if holder is None:
                    holder = AttributeNamespace(spec.namespace)
                    setattr(target, spec.namespace, holder)
            setattr(holder, spec.name, t)


__all__ = ["Model"]
