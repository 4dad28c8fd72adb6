"""Soft (particle-shape) contacts, mirroring the soft-contact part of
newton/_src/sim/contacts.py and the collision pipeline's soft contact
generation (newton/_src/sim/collide.py:1194-1228).

Arrays are torch tensors on the model's device: ``soft_contact_count`` (1,)
int32, ``soft_contact_particle`` / ``soft_contact_shape`` (max,) int32 and
``soft_contact_body_pos`` / ``soft_contact_body_vel`` /
``soft_contact_normal`` (max, 3) float32. ``Model.collide`` fills them on the
device in (particle, shape) order.
"""

from __future__ import annotations

import torch

from .. import _lib


class Contacts:
    """Soft contact buffers (rigid contacts are not part of this library)."""

    def __init__(self, soft_contact_max: int, particle_count: int, device):
        self.device = torch.device(device)
        self.soft_contact_max = int(soft_contact_max)
        m = max(self.soft_contact_max, 1)
        i32 = dict(dtype=torch.int32, device=self.device)
        f32 = dict(dtype=torch.float32, device=self.device)
        self.soft_contact_count = torch.zeros(1, **i32)
        self.soft_contact_particle = torch.zeros(m, **i32)
        self.soft_contact_shape = torch.zeros(m, **i32)
        self.soft_contact_body_pos = torch.zeros((m, 3), **f32)
        self.soft_contact_body_vel = torch.zeros((m, 3), **f32)
        self.soft_contact_normal = torch.zeros((m, 3), **f32)
        self.soft_contact_tids = None
        self.rigid_contact_max = 0
        self.force = None
        self._scratch = None
        self._particle_count = int(particle_count)
        if self.device.type == "cuda":
            n = _lib.load().nsph_soft_contacts_scratch_ints(self._particle_count)
            self._scratch = torch.zeros(n, **i32)

    def c_struct(self) -> _lib.NsphSoftContacts:
        """The nsph_soft_contacts view of these buffers."""
        return _lib.NsphSoftContacts(self.soft_contact_count.data_ptr(), self.soft_contact_particle.data_ptr(),
                                     self.soft_contact_shape.data_ptr(), self.soft_contact_body_pos.data_ptr(),
                                     self.soft_contact_body_vel.data_ptr(), self.soft_contact_normal.data_ptr(),
                                     self.soft_contact_max)

    def clear(self) -> None:
        self.soft_contact_count.zero_()


__all__ = ["Contacts"]
