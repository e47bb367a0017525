"""B200-native (sm_100a) Vertex Block Descent cloth path with Newton's model/solver interface.

Public names mirror ``newton`` for the cloth path: ``ModelBuilder``, ``Model``, ``State``,
``Control``, ``Contacts``, ``CollisionPipeline``, ``ParticleFlags``, ``ShapeFlags``, ``GeoType``
and ``solvers.SolverVBD``.
"""

from . import solvers
from .builder import ModelBuilder
from .collide import CollisionPipeline
from .coloring import ColoringAlgorithm
from .model import Contacts, Control, GeoType, Model, ModelFlags, ParticleFlags, ShapeFlags, State

__all__ = [
    "CollisionPipeline",
    "ColoringAlgorithm",
    "Contacts",
    "Control",
    "GeoType",
    "Model",
    "ModelBuilder",
    "ModelFlags",
    "ParticleFlags",
    "ShapeFlags",
    "State",
    "solvers",
]
