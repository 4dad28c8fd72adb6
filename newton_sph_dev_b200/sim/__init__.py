"""Particle data model: Model, State, Control, ModelBuilder."""

from .builder import ModelBuilder
from .control import Control
from .model import Model
from .state import AttributeNamespace, State

__all__ = ["AttributeNamespace", "Control", "Model", "ModelBuilder", "State"]
