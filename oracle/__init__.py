"""CPU oracle for the SQD hot path of t-imamichi/rqutils — TEST INFRASTRUCTURE ONLY.

This package is a NumPy restatement of the reference's algorithm, used as the checker by
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py``.  Nothing in the product package (``rqutils_b200``) imports it, and the product path
never falls back to it.

Each function cites the reference file:line it restates (paths relative to the rqutils project).

Parity status
-------------
The reference is pure Python on JAX and JAX is not installed in this image, so the reference's
own functions cannot be executed here, and the reference ships no golden vectors (its only test,
``tests/sqd.ipynb``, compares ``sqd`` against a dense ``eigh`` of the projected Qiskit matrix and
has no stored outputs).  The restatement is therefore pinned in two independent ways:

* against a dense Kronecker-product construction of every Pauli string (``oracle.dense``), which
  is independent of the symplectic bit tricks, and ``numpy.linalg.eigh`` of the projected matrix
  — the same check the reference's notebook performs;
* against the literal sort-based ``get_xsource`` algorithm (restated step by step), for bit-exact
  connectivity.

What is NOT pinned: the exact floating-point summation order of XLA's reductions inside
``ground_locg`` (``jnp.sum``/``jnp.linalg.norm``).  That boundary is "parity unpinned"; results
are compared with tolerances there.
"""
