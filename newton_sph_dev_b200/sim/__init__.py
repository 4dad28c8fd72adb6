"""Particle data model: Model, State, Control, ModelBuilder."""

from .builder import ModelBuilder
from .contacts import Contacts
from .control import Control
from .model import Model
from .state import AttributeNamespace, State

__all__ = ["AttributeNamespace", "Contacts", "Control", "Model", "ModelBuilder", "State"]
