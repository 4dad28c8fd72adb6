"""Scene construction for particles, mirroring the particle part of
newton/_src/sim/builder.py: __init__ (:795), add_particle (:7186-7230),
add_particles (:7232-7275), add_particle_grid (:8037-8130), begin_world /
end_world (:2815-2909), add_custom_attribute (:1266) and the particle part of
finalize (:9745, :9815-9855).

Particles are accumulated as numpy chunks instead of Python lists, so a
million-particle lattice is built in well under a second; the values, their
order and the jitter stream are the reference's.
"""

from __future__ import annotations

from collections.abc import Sequence
from typing import Any

import numpy as np
import torch

from ..geometry import ParticleFlags
from .model import Model


def quat_to_matrix(q) -> np.ndarray:
    """Rotation matrix (float32) of an (x, y, z, w) quaternion; columns are the
    rotated unit axes, computed with rotate(v) = v(2w^2-1) + 2w(u x v) + 2u(u.v)."""
    x, y, z, w = (np.float32(c) for c in q)
    u = np.array([x, y, z], dtype=np.float32)
    cols = []
    two = np.float32(2.0)
    for axis in np.eye(3, dtype=np.float32):
        r = axis * (two * w * w - np.float32(1.0)) + np.cross(u, axis) * w * two + u * np.dot(u, axis) * two
        cols.append(r.astype(np.float32))
    return np.stack(cols, axis=1)


class ModelBuilder:
    """Accumulates particles and worlds, then :meth:`finalize` makes a Model."""

    class CustomAttribute:
        """A custom attribute declaration (builder.py:516)."""

        def __init__(self, name: str, frequency=Model.AttributeFrequency.PARTICLE,
                     assignment=Model.AttributeAssignment.MODEL, dtype=torch.float32, default=0.0,
                     namespace: str | None = None, width: int = 1):
            self.name = name
            self.frequency = int(frequency)
            self.assignment = int(assignment)
            self.dtype = dtype
            self.default = default
            self.namespace = namespace
            self.width = width

        @property
        def key(self) -> str:
            return f"{self.namespace}:{self.name}" if self.namespace else self.name

    def __init__(self, up_axis: int = 2, gravity: float = -9.81):
        """
        Args:
            up_axis: 0 (x), 1 (y) or 2 (z, the default).
            gravity: magnitude of gravity along the up axis (default -9.81).
        """
        self.up_axis = int(up_axis)
        self.gravity: float = gravity
        self.world_count: int = 0
        self._current_world: int = -1
        self.world_gravity: list[tuple[float, float, float]] = []
        self.default_particle_radius = 0.1
        self.particle_max_velocity: float = 1e5
        self._chunks: list[dict[str, np.ndarray]] = []
        self._count = 0
        self.custom_attributes: dict[str, ModelBuilder.CustomAttribute] = {}
        self._requested_state_attributes: set[str] = set()

    # ------------------------------------------------------------------
    @property
    def up_vector(self) -> tuple[float, float, float]:
        v = [0.0, 0.0, 0.0]
        v[self.up_axis] = 1.0
        return tuple(v)

    @property
    def current_world(self) -> int:
        return self._current_world

    @property
    def particle_count(self) -> int:
        return self._count

    def _cat(self, key: str) -> np.ndarray:
        if not self._chunks:
            shape = {"q": (0, 3), "qd": (0, 3)}.get(key, (0,))
            dtype = {"flags": np.int32, "world": np.int32}.get(key, np.float64)
            return np.zeros(shape, dtype=dtype)
        return np.ascontiguousarray(np.concatenate([c[key] for c in self._chunks], axis=0))

    @property
    def particle_q(self) -> np.ndarray:
        return self._cat("q")

    @property
    def particle_qd(self) -> np.ndarray:
        return self._cat("qd")

    @property
    def particle_mass(self) -> np.ndarray:
        return self._cat("mass")

    @property
    def particle_radius(self) -> np.ndarray:
        return self._cat("radius")

    @property
    def particle_flags(self) -> np.ndarray:
        return self._cat("flags")

    @property
    def particle_world(self) -> np.ndarray:
        return self._cat("world")

    # ------------------------------------------------------------------
    def begin_world(self, label: str | None = None, attributes: dict[str, Any] | None = None, gravity=None) -> None:
        """Start a world context; particles added until :meth:`end_world`
        belong to it (builder.py:2815-2882)."""
        if self._current_world != -1:
            raise RuntimeError(
                f"Cannot begin a new world: already in world context (current_world={self._current_world}). "
                "Call end_world() first to close the current world context."
            )
        self._current_world = self.world_count
        self.world_count += 1
        if gravity is not None:
            self.world_gravity.append(tuple(float(g) for g in gravity))
        else:
            up = self.up_vector
            self.world_gravity.append((up[0] * self.gravity, up[1] * self.gravity, up[2] * self.gravity))

    def end_world(self) -> None:
        """Return to the global scope (builder.py:2884-2907)."""
        if self._current_world == -1:
            raise RuntimeError("Cannot end world: not currently in a world context (current_world is already -1).")
        self._current_world = -1

    def add_custom_attribute(self, attribute: ModelBuilder.CustomAttribute) -> None:
        """Declare a custom attribute (builder.py:1266)."""
        key = attribute.key
        if key in self.custom_attributes:
            old = self.custom_attributes[key]
            if (old.frequency, old.assignment, old.dtype) != (attribute.frequency, attribute.assignment, attribute.dtype):
                raise ValueError(f"Custom attribute '{key}' already registered with a different declaration")
            return
        self.custom_attributes[key] = attribute

    def request_state_attributes(self, *names: str) -> None:
        self._requested_state_attributes.update(names)

    # ------------------------------------------------------------------
    def _append(self, q, qd, mass, radius, flags) -> None:
        n = len(q)
        if n == 0:
            return
        self._chunks.append(
            {
                "q": np.ascontiguousarray(np.asarray(q, dtype=np.float64).reshape(n, 3)),
                "qd": np.ascontiguousarray(np.asarray(qd, dtype=np.float64).reshape(n, 3)),
                "mass": np.asarray(mass, dtype=np.float64).reshape(n),
                "radius": np.asarray(radius, dtype=np.float64).reshape(n),
                "flags": np.asarray(flags, dtype=np.int64).astype(np.int32).reshape(n),
                "world": np.full(n, self._current_world, dtype=np.int32),
            }
        )
        self._count += n

    def add_particle(self, pos, vel, mass: float, radius: float | None = None, flags: int = ParticleFlags.ACTIVE,
                     custom_attributes: dict[str, Any] | None = None) -> int:
        """Add one particle (builder.py:7186-7230). Zero mass makes it
        kinematic. Returns its index."""
        if radius is None:
            radius = self.default_particle_radius
        self._append([pos], [vel], [mass], [radius], [int(flags)])
        return self._count - 1

    def add_particles(self, pos, vel, mass, radius=None, flags=None,
                      custom_attributes: dict[str, Any] | None = None) -> None:
        """Add a group of particles (builder.py:7232-7275)."""
        n = len(pos)
        if radius is None:
            radius = np.full(n, self.default_particle_radius)
        if flags is None:
            flags = np.full(n, int(ParticleFlags.ACTIVE), dtype=np.int32)
        self._append(pos, vel, mass, radius, flags)

    def add_particle_grid(self, pos, rot, vel, dim_x: int, dim_y: int, dim_z: int, cell_x: float, cell_y: float,
                          cell_z: float, mass: float, jitter: float, radius_mean: float | None = None,
                          radius_std: float = 0.0, flags: list[int] | int | None = None,
                          custom_attributes: dict[str, Any] | None = None) -> None:
        """Add a jittered lattice (builder.py:8037-8130).

        Order: ``np.meshgrid`` with its default 'xy' indexing, so particle
        index = iy*(dim_x*dim_z) + ix*dim_z + iz. Jitter is
        ``(rng.random((N,3)) - 0.5) * jitter`` with
        ``rng = np.random.default_rng(42 + particle_count)``; radii are drawn
        from the same generator afterwards when ``radius_std > 0``.
        """
        px = np.arange(dim_x) * cell_x
        py = np.arange(dim_y) * cell_y
        pz = np.arange(dim_z) * cell_z
        points = np.stack(np.meshgrid(px, py, pz)).reshape(3, -1).T
        rot_mat = quat_to_matrix(rot)
        points = points @ np.array(rot_mat).reshape(3, 3).T + np.array(pos)
        velocity = np.broadcast_to(np.array(vel).reshape(1, 3), points.shape)
        rng = np.random.default_rng(42 + self._count)
        points += (rng.random(points.shape) - 0.5) * jitter
        if radius_mean is None:
            radius_mean = self.default_particle_radius
        radii = np.full(points.shape[0], fill_value=radius_mean, dtype=np.float64)
        if radius_std > 0.0:
            radii += rng.standard_normal(radii.shape) * radius_std
        n = points.shape[0]
        masses = np.full(n, mass, dtype=np.float64)
        if flags is None:
            fl = np.full(n, int(ParticleFlags.ACTIVE), dtype=np.int32)
        elif isinstance(flags, Sequence) or isinstance(flags, np.ndarray):
            fl = np.asarray(flags, dtype=np.int32)
            if fl.shape != (n,):
                raise ValueError(f"flags has {fl.size} values but {n} particles in grid")
        else:
            fl = np.full(n, int(flags), dtype=np.int32)
        self._append(points, velocity, masses, radii, fl)

    # ------------------------------------------------------------------
    def finalize(self, device: str | torch.device = "cuda:0", requires_grad: bool = False) -> Model:
        """Build the Model on `device` (particle part of builder.py:9745-9855
        and gravity :10655-10668)."""
        device = torch.device(device)
        self.world_count = max(1, self.world_count)
        m = Model(device)
        m.requires_grad = requires_grad
        m.world_count = self.world_count
        m.up_axis = self.up_axis
        n = self._count
        q = np.ascontiguousarray(self.particle_q, dtype=np.float32)
        qd = np.ascontiguousarray(self.particle_qd, dtype=np.float32)
        ms = self.particle_mass.astype(np.float32)
        inv = np.divide(1.0, ms, out=np.zeros_like(ms), where=ms != 0.0).astype(np.float32)
        radius = self.particle_radius.astype(np.float32)
        m.particle_q = torch.from_numpy(q).to(device)
        m.particle_qd = torch.from_numpy(qd).to(device)
        m.particle_mass = torch.from_numpy(ms).to(device)
        m.particle_inv_mass = torch.from_numpy(inv).to(device)
        m.particle_radius = torch.from_numpy(radius).to(device)
        m.particle_flags = torch.from_numpy(self.particle_flags.astype(np.int32)).to(device)
        world = self.particle_world.astype(np.int32)
        m.particle_world = torch.from_numpy(world).to(device)
        m.particle_world_start = torch.from_numpy(self._world_starts(world)).to(device)
        m.particle_max_radius = float(np.max(self.particle_radius)) if n > 0 else 0.0
        m.particle_max_velocity = self.particle_max_velocity
        m.particle_count = n
        if self.world_gravity:
            g = np.asarray(self.world_gravity, dtype=np.float32)
            if len(g) < self.world_count:
                up = self.up_vector
                pad = np.tile(np.asarray([u * self.gravity for u in up], dtype=np.float32), (self.world_count - len(g), 1))
                g = np.concatenate([g, pad])
        else:
            gv = [u * self.gravity for u in self.up_vector]
            g = np.asarray([gv] * self.world_count, dtype=np.float32)
        m.gravity = torch.from_numpy(g.reshape(self.world_count, 3)).to(device)
        for key, attr in self.custom_attributes.items():
            m.custom_attributes[key] = Model.CustomAttributeSpec(
                attr.name, attr.namespace, attr.frequency, attr.assignment, attr.dtype, attr.width, attr.default
            )
        m._requested_state_attributes = set(self._requested_state_attributes)
        if n > 1 and m.particle_max_radius > 0.0 and device.type == "cuda":
            from ..hashgrid import HashGrid

            m.particle_grid = HashGrid(128, 128, 128, device=device)
        return m

    def _world_starts(self, world: np.ndarray) -> np.ndarray:
        """particle_world_start (model.py:172-178): per-world start indices,
        then the start of the global particles, then the total."""
        wc = self.world_count
        counts = np.bincount(world[world >= 0], minlength=wc) if len(world) else np.zeros(wc, dtype=np.int64)
        starts = np.zeros(wc + 2, dtype=np.int32)
        starts[1 : wc + 1] = np.cumsum(counts[:wc])
        starts[wc] = int(np.sum(counts[:wc]))
        starts[wc + 1] = len(world)
        return starts


__all__ = ["ModelBuilder", "quat_to_matrix"]
