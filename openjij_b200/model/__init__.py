"""Models of the sampler path: BinaryQuadraticModel and the lattice models
(ChimeraModel, KingGraph) of openjij/model/."""
from . import chimera_model, king_graph  # noqa: F401
from .model import BinaryQuadraticModel, make_BinaryQuadraticModel  # noqa: F401

__all__ = ["BinaryQuadraticModel", "make_BinaryQuadraticModel"]
