"""Particle flags, as in newton/_src/geometry/flags.py:8-14."""

from enum import IntEnum


class ParticleFlags(IntEnum):
    """Flags for particle properties."""

    ACTIVE = 1 << 0
    """Indicates that the particle is active."""


__all__ = ["ParticleFlags"]
