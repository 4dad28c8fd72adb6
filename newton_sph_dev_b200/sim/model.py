"""Static particle model, mirroring the particle part of
newton/_src/sim/model.py (fields :140-178, gravity :631, particle_count :691,
state() :827-878, control() :880, set_gravity() :923-956), the soft-contact
material (:613-623) and contacts() / collide() (:970-1022) for static
shapes.

Storage is torch tensors on the model's device (the reference uses
``wp.array``); vec3 arrays have shape ``(N, 3)`` float32.
"""

from __future__ import annotations

import ctypes
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
        self.soft_contact_ke: float = 1.0e3
        """Particle side of the particle-shape contact stiffness [N/m]."""
        self.soft_contact_kd: float = 10.0
        self.soft_contact_kf: float = 1.0e3
        self.soft_contact_mu: float = 0.5
        self.soft_contact_restitution: float = 0.0
        """Restitution of particle-shape contacts (XPBD with enable_restitution)."""
        self.shape_type: torch.Tensor | None = None
        """GeoType per shape, int32."""
        self.shape_body: torch.Tensor | None = None
        """Body per shape (-1: static), int32."""
        self.shape_transform: torch.Tensor | None = None
        """World transform per shape, (shape_count, 7) float32: position, then quaternion (x, y, z, w)."""
        self.shape_scale: torch.Tensor | None = None
        self.shape_flags: torch.Tensor | None = None
        self.shape_world: torch.Tensor | None = None
        self.shape_material_ke: torch.Tensor | None = None
        self.shape_material_kd: torch.Tensor | None = None
        self.shape_material_kf: torch.Tensor | None = None
        self.shape_material_ka: torch.Tensor | None = None
        self.shape_material_mu: torch.Tensor | None = None
        self.shape_material_restitution: torch.Tensor | None = None
        self.shape_label: list[str] = []
        self._shapes: list[dict] = []
        self._shapes_dev: torch.Tensor | None = None
        self._contacts = None
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

    # ------------------------------------------------------------------
    # static shapes and soft contacts
    def _set_shapes(self, shapes: list[dict]) -> None:
        """Shape arrays of the finalized model (static shapes only)."""
        self._shapes = [dict(s) for s in shapes]
        self.shape_count = len(shapes)
        d = self.device
        self.shape_label = [s["label"] for s in shapes]
        self.shape_type = torch.tensor([s["type"] for s in shapes], dtype=torch.int32, device=d)
        self.shape_body = torch.full((len(shapes),), -1, dtype=torch.int32, device=d)
        self.shape_transform = torch.tensor([list(s["pos"]) + list(s["rot"]) for s in shapes], dtype=torch.float32,
                                            device=d).reshape(-1, 7)
        self.shape_scale = torch.tensor([list(s["scale"]) for s in shapes], dtype=torch.float32,
                                        device=d).reshape(-1, 3)
        self.shape_flags = torch.tensor([s["flags"] for s in shapes], dtype=torch.int32, device=d)
        self.shape_world = torch.tensor([s["world"] for s in shapes], dtype=torch.int32, device=d)
        for k in ("ke", "kd", "kf", "ka", "mu", "restitution"):
            setattr(self, f"shape_material_{k}",
                    torch.tensor([s[k] for s in shapes], dtype=torch.float32, device=d))
        self._shapes_dev = None

    def shapes_device(self) -> torch.Tensor | None:
        """The shapes as a device array of nsph_shape records (rebuilt from
        the shape_* arrays, so edits to them take effect)."""
        if not self.shape_count:
            return None
        from .. import _lib

        arr = (_lib.NsphShape * self.shape_count)()
        tf = self.shape_transform.detach().cpu().numpy()
        sc = self.shape_scale.detach().cpu().numpy()
        ty = self.shape_type.cpu().numpy()
        fl = self.shape_flags.cpu().numpy()
        wo = self.shape_world.cpu().numpy()
        mats = {k: getattr(self, f"shape_material_{k}").detach().cpu().numpy() for k in ("ke", "kd", "kf", "mu")}
        for i in range(self.shape_count):
            arr[i].type = int(ty[i])
            arr[i].flags = int(fl[i])
            arr[i].world = int(wo[i])
            arr[i].pos[:] = [float(v) for v in tf[i, :3]]
            arr[i].rot[:] = [float(v) for v in tf[i, 3:7]]
            arr[i].scale[:] = [float(v) for v in sc[i]]
            for k in ("ke", "kd", "kf", "mu"):
                setattr(arr[i], k, float(mats[k][i]))
        host = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8)
        self._shapes_dev = host.to(self.device)
        return self._shapes_dev

    def contacts(self, soft_contact_max: int | None = None):
        """A Contacts object for this model (model.py:970-994); its soft
        contact capacity defaults to shape_count * particle_count, as in the
        reference's collision pipeline."""
        from .contacts import Contacts

        mx = self.shape_count * self.particle_count if soft_contact_max is None else int(soft_contact_max)
        return Contacts(mx, self.particle_count, self.device)

    def collide(self, state, contacts=None, soft_contact_margin: float = 0.01):
        """Generate the soft contacts of the particles of `state` with the
        model's static shapes (model.py:996-1022; create_soft_contacts,
        newton/_src/geometry/kernels.py:1001-1140), on the device, in
        (particle, shape) order. Returns the contacts."""
        from .. import _lib

        if contacts is None:
            if self._contacts is None:
                self._contacts = self.contacts()
            contacts = self._contacts
        if not self.shape_count or not self.particle_count or contacts.soft_contact_max == 0:
            contacts.clear()
            return contacts
        if self._shapes_dev is None:
            self.shapes_device()
        c = contacts.c_struct()
        st = _lib.load().nsph_soft_contacts_create(
            self._shapes_dev.data_ptr(), self.shape_count, self.particle_count, state.particle_q.data_ptr(),
            self.particle_radius.data_ptr(), self.particle_flags.data_ptr(), self.particle_world.data_ptr(),
            float(soft_contact_margin), ctypes.byref(c), contacts._scratch.data_ptr(), _lib.stream_handle(self.device))
        _lib.check(st, "collide")
        return contacts

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
