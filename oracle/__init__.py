"""CPU oracle for the SQD hot path of t-imamichi/rqutils — TEST INFRASTRUCTURE ONLY.

This package is a NumPy restatement of the reference's algorithm, used as the checker by
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py``.  Nothing in the product package (``rqutils_b200``) imports it, and the product path
never falls back to it.

Each function cites the reference file:line it restates (paths relative to the rqutils project).

Parity status
-------------
Pinned to the reference's own execution.  The reference is pure Python on JAX, which is not
installed in this image; ``tests/golden/make_reference_golden.py`` imports the UNMODIFIED
reference modules through a NumPy stand-in for the JAX subset they use
(``tests/golden/jax_stand_in``) and records their outputs as ``tests/golden/reference_*.npz``.
``tests/test_reference_golden.py`` and ``tests/test_oracle_cpu_baseline.py`` check this
restatement against them: Pauli tables, uniquified rows and indices, source indices, group
diagonals and start indices bit for bit; matvecs, energies and small eigenpairs to written
tolerances.  Also kept: the independent dense Kronecker-product construction
(``oracle.dense``) with ``numpy.linalg.eigh``, the check of the reference's notebook.

What is NOT pinned: XLA's floating-point summation order inside ``jnp.sum`` /
``jnp.linalg.norm`` (the stand-in sums in NumPy's order); results are compared with tolerances
there.
"""
