"""Solver notification flags, as in newton/_src/solvers/flags.py:1-60."""

from enum import IntEnum


class SolverNotifyFlags(IntEnum):
    """Flags telling a solver which parts of the model changed
    (``solver.notify_model_changed(flags)``)."""

    JOINT_PROPERTIES = 1 << 0
    JOINT_DOF_PROPERTIES = 1 << 1
    BODY_PROPERTIES = 1 << 2
    BODY_INERTIAL_PROPERTIES = 1 << 3
    SHAPE_PROPERTIES = 1 << 4
    MODEL_PROPERTIES = 1 << 5
    """Model global properties (gravity, particle_max_velocity, ...) changed."""
    CONSTRAINT_PROPERTIES = 1 << 6
    TENDON_PROPERTIES = 1 << 7
    ACTUATOR_PROPERTIES = 1 << 8
    ALL = (
        JOINT_PROPERTIES
        | JOINT_DOF_PROPERTIES
        | BODY_PROPERTIES
        | BODY_INERTIAL_PROPERTIES
        | SHAPE_PROPERTIES
        | MODEL_PROPERTIES
        | CONSTRAINT_PROPERTIES
        | TENDON_PROPERTIES
        | ACTUATOR_PROPERTIES
    )


__all__ = ["SolverNotifyFlags"]
