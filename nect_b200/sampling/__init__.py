"""Ray sampling: geometry, the ct_sampling drop-in and the Projector."""
from . import ct_sampling
from .geometry import Geometry
from .projector import Projector

__all__ = ["Geometry", "Projector", "ct_sampling"]
