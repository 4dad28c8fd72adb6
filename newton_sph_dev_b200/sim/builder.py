"""Scene construction for particles, mirroring the particle part of
newton/_src/sim/builder.py: __init__ (:795), add_particle (:7186-7230),
add_particles (:7232-7275), add_particle_grid (:8037-8130), begin_world /
end_world (:2815-2909), add_custom_attribute (:1266) and the particle part of
finalize (:9745, :9815-9855); and static collision shapes for particle
contacts: ShapeConfig (:231), add_shape_plane / add_ground_plane /
add_shape_sphere / add_shape_box (:5611-5891) for shapes without a body.

Particles are accumulated as numpy chunks instead of Python lists, so a
million-particle lattice is built in well under a second; the values, their
order and the jitter stream are the reference's.
"""

from __future__ import annotations

from collections.abc import Sequence
from typing import Any

import numpy as np
import torch

from ..geometry import GeoType, ParticleFlags, ShapeFlags
from .model import Model

_AXES = {"X": 0, "Y": 1, "Z": 2}


def _axis_index(axis) -> int:
    """0/1/2 from an int or "X"/"Y"/"Z" (newton's Axis)."""
    if isinstance(axis, str):
        return _AXES[axis.upper()]
    return int(axis)


def quat_between_vectors(a, b) -> tuple[float, float, float, float]:
    """Unit quaternion (x, y, z, w) rotating unit vector a onto unit vector b:
    axis a x b, half-angle from a.b (the half-vector construction); a
    rotation by pi about an axis orthogonal to a when b = -a."""
    a = np.asarray(a, dtype=np.float64) / np.linalg.norm(a)
    b = np.asarray(b, dtype=np.float64) / np.linalg.norm(b)
    c = float(np.dot(a, b))
    if c < -1.0 + 1e-12:
        helper = np.array([1.0, 0.0, 0.0]) if abs(a[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
        axis = np.cross(a, helper)
        axis /= np.linalg.norm(axis)
        return (float(axis[0]), float(axis[1]), float(axis[2]), 0.0)
    axis = np.cross(a, b)
    s = np.sqrt(2.0 * (1.0 + c))
    return (float(axis[0] / s), float(axis[1] / s), float(axis[2] / s), float(0.5 * s))


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

    class ShapeConfig:
        """Physical and collision properties of a shape (builder.py:231-300):
        the contact material ke / kd / kf / ka / mu, restitution, and whether
        the shape collides with particles."""

        def __init__(self, ke: float = 2.5e3, kd: float = 100.0, kf: float = 1000.0, ka: float = 0.0,
                     mu: float = 1.0, restitution: float = 0.0, density: float = 1000.0,
                     has_shape_collision: bool = True, has_particle_collision: bool = True,
                     is_visible: bool = True, is_site: bool = False):
            self.ke = ke
            self.kd = kd
            self.kf = kf
            self.ka = ka
            self.mu = mu
            self.restitution = restitution
            self.density = density
            self.has_shape_collision = has_shape_collision
            self.has_particle_collision = has_particle_collision
            self.is_visible = is_visible
            self.is_site = is_site

        def copy(self) -> "ModelBuilder.ShapeConfig":
            c = ModelBuilder.ShapeConfig()
            c.__dict__.update(self.__dict__)
            return c

        def mark_as_site(self) -> None:
            """A site: no shape or particle collision, zero density (builder.py:389-403)."""
            self.is_site = True
            self.has_shape_collision = False
            self.has_particle_collision = False
            self.density = 0.0

        @property
        def flags(self) -> int:
            f = int(ShapeFlags.VISIBLE) if self.is_visible else 0
            f |= int(ShapeFlags.COLLIDE_SHAPES) if self.has_shape_collision else 0
            f |= int(ShapeFlags.COLLIDE_PARTICLES) if self.has_particle_collision else 0
            f |= int(ShapeFlags.SITE) if self.is_site else 0
            return f

    def __init__(self, up_axis: int | str = 2, gravity: float = -9.81):
        """
        Args:
            up_axis: 0 / "X", 1 / "Y" or 2 / "Z" (the default).
            gravity: magnitude of gravity along the up axis (default -9.81).
        """
        self.up_axis = _axis_index(up_axis)
        self.default_shape_cfg = ModelBuilder.ShapeConfig()
        self.shapes: list[dict] = []
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
    # static collision shapes (body -1)
    def add_shape(self, body: int, type: int, xform=None, cfg: ShapeConfig | None = None, scale=(1.0, 1.0, 1.0),
                  is_static: bool = True, label: str | None = None, **_ignored) -> int:
        """Add a collision shape (builder.py add_shape). Only shapes without a
        body (body == -1) are supported: rigid bodies are outside this
        library."""
        if int(body) != -1:
            raise NotImplementedError("only static shapes (body=-1) are supported; rigid bodies are not part of the "
                                      "particle path")
        cfg = cfg if cfg is not None else self.default_shape_cfg
        if xform is None:
            xform = ((0.0, 0.0, 0.0), (0.0, 0.0, 0.0, 1.0))
        pos, rot = xform
        self.shapes.append(dict(type=int(type), flags=cfg.flags, world=self._current_world,
                                pos=tuple(float(v) for v in pos), rot=tuple(float(v) for v in rot),
                                scale=tuple(float(v) for v in scale), ke=cfg.ke, kd=cfg.kd, kf=cfg.kf, ka=cfg.ka,
                                mu=cfg.mu, restitution=cfg.restitution, label=label or f"shape_{len(self.shapes)}"))
        return len(self.shapes) - 1

    def add_shape_plane(self, plane=(0.0, 0.0, 1.0, 0.0), xform=None, width: float = 10.0, length: float = 10.0,
                        body: int = -1, cfg: ShapeConfig | None = None, color=None, label: str | None = None,
                        custom_attributes=None) -> int:
        """A plane (builder.py:5611-5674): with xform None it comes from the
        plane equation a x + b y + c z + d = 0 (normal (a, b, c), offset
        -d/|n| along it); the collision normal is the local +Z. width /
        length 0 make it infinite for collision."""
        if xform is None:
            normal = np.asarray(plane[:3], dtype=np.float64)
            norm = np.linalg.norm(normal)
            normal = normal / norm
            pos = -(plane[3] / norm) * normal
            xform = (tuple(pos), quat_between_vectors((0.0, 0.0, 1.0), normal))
        return self.add_shape(body, GeoType.PLANE, xform, cfg, (width, length, 0.0), label=label)

    def add_ground_plane(self, height: float = 0.0, cfg: ShapeConfig | None = None, color=None,
                         label: str | None = None) -> int:
        """An infinite plane through height along the up axis (builder.py:5676-5701)."""
        return self.add_shape_plane(plane=(*self.up_vector, -height), width=0.0, length=0.0, cfg=cfg,
                                    label=label or "ground_plane")

    def _shape_cfg(self, cfg, as_site: bool):
        """The shape's config; a site gets a copy marked as one (as the
        reference's add_shape_* do with as_site)."""
        if not as_site:
            return cfg
        cfg = (cfg if cfg is not None else self.default_shape_cfg).copy()
        cfg.mark_as_site()
        return cfg

    def add_shape_sphere(self, body: int, xform=None, radius: float = 1.0, cfg: ShapeConfig | None = None,
                         as_site: bool = False, color=None, label: str | None = None, custom_attributes=None) -> int:
        """A sphere of the given radius centred at xform (builder.py:5703)."""
        return self.add_shape(body, GeoType.SPHERE, xform, self._shape_cfg(cfg, as_site), (radius, 0.0, 0.0),
                              label=label)

    def add_shape_box(self, body: int, xform=None, hx: float = 0.5, hy: float = 0.5, hz: float = 0.5,
                      cfg: ShapeConfig | None = None, as_site: bool = False, color=None, label: str | None = None,
                      custom_attributes=None) -> int:
        """A box with half extents (hx, hy, hz) at xform (builder.py:5842)."""
        return self.add_shape(body, GeoType.BOX, xform, self._shape_cfg(cfg, as_site), (hx, hy, hz), label=label)

    def add_shape_ellipsoid(self, body: int, xform=None, rx: float = 1.0, ry: float = 0.75, rz: float = 0.5,
                            cfg: ShapeConfig | None = None, as_site: bool = False, color=None,
                            label: str | None = None, custom_attributes=None, **kwargs) -> int:
        """An ellipsoid with semi-axes (rx, ry, rz) along its local axes
        (builder.py:5747-5790). Its particle contacts use the reference's
        approximate SDF k0 (k0 - 1) / k1."""
        return self.add_shape(body, GeoType.ELLIPSOID, xform, self._shape_cfg(cfg, as_site), (rx, ry, rz),
                              label=label)

    def add_shape_capsule(self, body: int, xform=None, radius: float = 1.0, half_height: float = 0.5,
                          cfg: ShapeConfig | None = None, as_site: bool = False, color=None,
                          label: str | None = None, custom_attributes=None) -> int:
        """A capsule along its local Z axis: a cylinder of the given radius
        and half height with hemispherical ends (builder.py:5892-5943)."""
        return self.add_shape(body, GeoType.CAPSULE, xform, self._shape_cfg(cfg, as_site), (radius, half_height, 0.0),
                              label=label)

    def add_shape_cylinder(self, body: int, xform=None, radius: float = 1.0, half_height: float = 0.5,
                           cfg: ShapeConfig | None = None, as_site: bool = False, color=None,
                           label: str | None = None, custom_attributes=None) -> int:
        """A cylinder along its local Z axis (builder.py:5945-5996)."""
        return self.add_shape(body, GeoType.CYLINDER, xform, self._shape_cfg(cfg, as_site),
                              (radius, half_height, 0.0), label=label)

    def add_shape_cone(self, body: int, xform=None, radius: float = 1.0, half_height: float = 0.5,
                       cfg: ShapeConfig | None = None, as_site: bool = False, color=None, label: str | None = None,
                       custom_attributes=None) -> int:
        """A cone along its local Z axis, base of the given radius at
        -half_height and apex at +half_height (builder.py:5998-6050)."""
        return self.add_shape(body, GeoType.CONE, xform, self._shape_cfg(cfg, as_site), (radius, half_height, 0.0),
                              label=label)

    @property
    def shape_count(self) -> int:
        return len(self.shapes)

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
        m._set_shapes(self.shapes)
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


__all__ = ["ModelBuilder", "quat_between_vectors", "quat_to_matrix"]
