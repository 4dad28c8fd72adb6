"""Control inputs, mirroring newton/_src/sim/control.py:9-86.

A particle fluid uses none of them; the object exists so that
``solver.step(state_in, state_out, control, contacts, dt)`` keeps the
reference's signature.
"""

from __future__ import annotations


class Control:
    """Time-varying control data (joint/tri/tet/muscle inputs: all None for
    a particle-only model)."""

    def __init__(self) -> None:
        self.joint_f = None
        self.joint_target_pos = None
        self.joint_target_vel = None
        self.joint_act = None
        self.tri_activations = None
        self.tet_activations = None
        self.muscle_activations = None

    def clear(self) -> None:
        """Reset the control inputs to zero."""
        for name in ("joint_f", "joint_target_pos", "joint_target_vel", "joint_act", "tri_activations",
                     "tet_activations", "muscle_activations"):
            val = getattr(self, name)
            if val is not None:
                val.zero_()


__all__ = ["Control"]
