"""Geometry enums: particle flags (newton/_src/geometry/flags.py:8-14),
shape flags (flags.py:18-33) and shape types (newton/_src/geometry/types.py:
38-80), with the reference's integer values so user code passes the same
numbers."""

from enum import IntEnum


class ParticleFlags(IntEnum):
    """Flags for particle properties."""

    ACTIVE = 1 << 0
    """Indicates that the particle is active."""


class ShapeFlags(IntEnum):
    """Flags for shape properties."""

    VISIBLE = 1 << 0
    COLLIDE_SHAPES = 1 << 1
    COLLIDE_PARTICLES = 1 << 2
    """The shape makes soft contacts with particles."""
    SITE = 1 << 3


class GeoType(IntEnum):
    """Shape types. This library makes particle contacts with PLANE, SPHERE,
    BOX, CAPSULE, CYLINDER, CONE and ELLIPSOID shapes that belong to no
    body."""

    NONE = 0
    PLANE = 1
    HFIELD = 2
    SPHERE = 3
    CAPSULE = 4
    ELLIPSOID = 5
    CYLINDER = 6
    BOX = 7
    MESH = 8
    CONE = 9
    CONVEX_MESH = 10
    GAUSSIAN = 11


__all__ = ["GeoType", "ParticleFlags", "ShapeFlags"]
