"""B200-native (sm_100a) implementation of the sample-based quantum diagonalization hot path of
rqutils: Pauli-sum preprocessing, subspace build, the matrix-free Pauli-sum matvec over a sorted
subspace of computational-basis bitstrings, and the single-vector LOCG/LOBPCG ground-state
solver — all as CUDA kernels behind the C ABI in ``include/sqd_b200.h``.
"""
from . import _lib
from .paulis.symplectic import PauliSumXZ
from .sqd import (SQDOptions, SQDOperator, Subspace, sqd, run_sqd, hproj, uniquify_states,
                  get_xsource, get_diagonal)
from .ground_locg import ground_locg

# The shared library is mapped by the first call that needs it (``_lib.load()``, which raises
# ImportError when the library is missing), so importing the package for its pure-Python parts
# (the seeded workload generators, the option types) maps no native code.

__all__ = ['PauliSumXZ', 'SQDOptions', 'SQDOperator', 'Subspace', 'sqd', 'run_sqd', 'hproj',
           'uniquify_states', 'get_xsource', 'get_diagonal', 'ground_locg']
