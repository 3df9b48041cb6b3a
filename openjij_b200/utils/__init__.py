"""Helpers of the reference's ``openjij.utils`` used with the lattice models."""
from .graph_utils import chimera_to_ind, qubo_to_ising

__all__ = ["chimera_to_ind", "qubo_to_ising"]
