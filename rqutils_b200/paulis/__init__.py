"""Pauli-sum containers (``rqutils.paulis`` counterpart, symplectic representation only)."""
from .symplectic import PauliSumXZ

__all__ = ['PauliSumXZ']
