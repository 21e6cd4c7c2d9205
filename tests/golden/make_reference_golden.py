"""Writes ``reference_*.npz`` in this folder from the reference's OWN code (test infrastructure).

Run in a container that holds the rqutils checkout (``python -m tests.golden.make_reference_golden
[reference root]``; default root ``/root/reference``).  The unmodified modules
``rqutils/sqd.py``, ``rqutils/ground_locg.py`` and ``rqutils/paulis/symplectic.py`` are imported
through the NumPy stand-in for JAX (``reference_loader.py``, ``jax_stand_in/``) and called
through their public functions; nothing here restates their algorithms.  The inputs come from
the seeded generators of ``rqutils_b200.workloads`` (pure Python, no native code).

What the reference itself allows, and so what the fixtures hold:

* ``PauliSumXZ.from_paulisum``, ``uniquify_states``, ``get_xsource`` (both input orders),
  ``get_diagonal`` and every cached/uncached matvec ``run_sqd`` assembles: for real and complex
  Pauli sums.  The matvec, the start index and the solver's arguments are captured by replacing
  the ``ground_locg`` name that ``rqutils.sqd`` calls with a recorder (the call's arguments are
  what ``run_sqd`` built).
* ``sqd`` and ``ground_locg`` solves: real Hamiltonians only.  For complex vectors the
  reference's ``lax.cond`` in ``body_iter1`` (ground_locg.py:314-318) returns ``jnp.zeros(2)``
  (float64) in one branch and a complex ``kappa`` in the other, which JAX rejects at trace time
  ("must have identical types"); the stand-in applies the same check.
* ``sqd`` is called with an explicit ``options``: with ``options=None`` the reference
  dereferences ``options.return_eigvec`` (sqd.py:262) before any default is set.
* ``eigenpair_2x2`` / ``eigenpair_3x3`` on random, degenerate and near-degenerate matrices.

Floating-point outputs carry NumPy's summation order instead of XLA's (see the stand-in's
README); integer outputs are the reference's exactly.
"""
import logging
import os
import sys
import time
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from tests.golden import reference_loader            # noqa: E402
from rqutils_b200 import workloads as W              # noqa: E402  (pure-Python generators)


def bits_of(values, n):
    """uint64 states (bit q = qubit q) -> binary [N, n] rows in Qiskit order (last column =
    qubit 0), the ``states`` argument of ``sqd``."""
    values = np.asarray(values, dtype=np.uint64)
    shifts = np.arange(n - 1, -1, -1, dtype=np.uint64)
    return ((values[:, None] >> shifts[None, :]) & np.uint64(1)).astype(np.uint8)


def pack(bits):
    """The packing of sqd.py:255 (pad bit first, big-endian bytes), written with NumPy's
    per-axis pad list."""
    return np.packbits(np.pad(bits.astype(np.uint8), ((0, 0), (1, 0))), axis=1)


def labels_array(labels):
    return np.array([s.encode() for s in labels], dtype='S')


class _Stop(Exception):
    pass


class Recorder:
    """Stands in for the ``ground_locg`` that ``rqutils.sqd.run_sqd`` calls: records the start
    index, applies the assembled matvec to probe vectors and optionally runs the real solver."""

    def __init__(self, R):
        self.R = R
        self.real = R.ground_locg.ground_locg
        R.sqd.ground_locg = self

    def arm(self, probes, solve):
        self.probes = probes
        self.solve = solve
        self.vinit = None
        self.hv = None
        self.niter = None

    def __call__(self, matvec, xinit, args=(), orth=(), maxiter=1000, tol=None, vspace=None,
                 log_level=logging.WARNING):
        self.vinit = int(np.asarray(xinit))
        self.hv = (np.stack([np.asarray(matvec(p, *args)) for p in self.probes])
                   if len(self.probes) else None)
        if not self.solve:
            raise _Stop()
        e, v, it = self.real(matvec, xinit, args=args, orth=orth, maxiter=maxiter, tol=tol,
                             vspace=vspace, log_level=log_level)
        self.niter = int(it)
        return e, v, it


def run_sqd_capture(R, rec, ham, bits, states_size, cache, probes, solve=False, maxiter=1000,
                    tol=None):
    opts = R.sqd.SQDOptions(cache_strategy=cache, locg_maxiter=maxiter, locg_tol=tol)
    rec.arm(probes, solve)
    try:
        out = R.sqd.sqd(ham, bits, states_size=states_size, options=opts)
    except _Stop:
        out = None
    return out


# ------------------------------------------------------------------------------------- cases
def paulis_case(R):
    rng = np.random.default_rng(101)
    x, z, c = W.random_pauli_sum(10, 80, rng)
    labels = W.labels_from_xz(x, z, 10)
    # explicit duplicates, a zero coefficient, a cancelling pair, lower-case letters
    labels += [labels[3], labels[7], 'IIIIIIIIII', 'XYZIIIIIIZ', 'XYZIIIIIIZ', 'xyziiiiiiz']
    coeffs = np.concatenate([c, [0.5, -0.25, 1.5, 0.0, 2.0, -2.0]])
    cplx = coeffs + 1j * rng.standard_normal(coeffs.shape[0]) * 0.1
    P = R.symplectic.PauliSumXZ
    out = {'labels': labels_array(labels), 'coeffs': coeffs, 'coeffs_complex': cplx}
    for tag, arg, kw in (('real_pad', coeffs, dict(add_padding=True)),
                         ('real_nopad', coeffs, dict()),
                         ('cplx_nopad', cplx, dict()),
                         ('cplx_forcereal_pad', cplx, dict(force_real=True, add_padding=True))):
        with warnings.catch_warnings(record=True) as caught:
            warnings.simplefilter('always')
            h = P.from_paulisum((labels, list(arg)), **kw)
        out[f'{tag}_x'], out[f'{tag}_z'], out[f'{tag}_c'] = h.x, h.z, h.c
        out[f'{tag}_warned'] = np.array(any('imaginary' in str(w.message) for w in caught))
    return out


def subspace_case(R, rec):
    """10 qubits: complex Pauli sum, repeated and unsorted samples, fill rows."""
    rng = np.random.default_rng(303)
    n = 10
    x, z, c = W.random_pauli_sum(n, 70, rng)
    labels = W.labels_from_xz(x, z, n)
    distinct = rng.choice(1 << n, size=180, replace=False).astype(np.uint64)
    repeats = rng.choice(distinct, size=60)
    samples = np.concatenate([distinct, repeats])
    rng.shuffle(samples)
    bits = bits_of(samples, n)
    sp = pack(bits)
    ham = R.symplectic.PauliSumXZ.from_paulisum((labels, list(c)), force_real=True,
                                                add_padding=True)
    out = {'labels': labels_array(labels), 'coeffs': c, 'bits': bits, 'packed': sp,
           'x': ham.x, 'z': ham.z, 'c': ham.c}
    for tag, size in (('plus', 200), ('exact', 180), ('minus', 170), ('all', sp.shape[0])):
        su, idx = R.sqd.uniquify_states(sp, size, return_indices=True)
        out[f'uniq_{tag}'] = np.asarray(su)
        out[f'uniq_{tag}_idx'] = np.asarray(idx)
    su = np.asarray(R.sqd.uniquify_states(sp, 200))
    out['xsource'] = np.stack([np.asarray(R.sqd.get_xsource(xx, su)) for xx in ham.x])
    out['diagonal'] = np.stack([np.asarray(R.sqd.get_diagonal(zz, cc, su))
                                for zz, cc in zip(ham.z, ham.c)])
    # unsorted unique rows, no fill rows
    uniq_bits = bits_of(distinct, n)
    usp = pack(uniq_bits)
    out['unsorted_bits'] = uniq_bits
    out['xsource_unsorted'] = np.stack([np.asarray(R.sqd.get_xsource(xx, usp,
                                                                     sorted_input=False))
                                        for xx in ham.x])
    # run_sqd on all 240 samples with states_size 260: 180 unique rows and 80 fill rows
    probes = np.stack([rng.standard_normal(260) + 1j * rng.standard_normal(260)
                       for _ in range(2)])
    out['probes'] = probes
    for cache in ((1, 0), (1, 2), (0, 0), (0, 2)):
        run_sqd_capture(R, rec, (labels, list(c)), bits, 260, cache, probes)
        out[f'hv_{cache[0]}{cache[1]}'] = rec.hv
        out[f'vinit_{cache[0]}{cache[1]}'] = np.array(rec.vinit)
    return out


def c1_case(R, rec):
    """The 16-qubit random Pauli sum on 2000 weight-8 strings (complex): the assembled matvec
    and start index (a complex solve is rejected by the reference, see the module docstring)."""
    wl = W.c1(0)
    labels = wl.labels
    bits = bits_of(wl.states, 16)
    rng = np.random.default_rng(404)
    probes = np.stack([rng.standard_normal(2000) + 1j * rng.standard_normal(2000)])
    out = {'probes': probes}
    for cache in ((1, 0), (1, 2)):
        run_sqd_capture(R, rec, (labels, list(wl.coeffs)), bits, None, cache, probes)
        out[f'hv_{cache[0]}{cache[1]}'] = rec.hv
        out[f'vinit_{cache[0]}{cache[1]}'] = np.array(rec.vinit)
    ham = R.symplectic.PauliSumXZ.from_paulisum((labels, list(wl.coeffs)), force_real=True,
                                                add_padding=True)
    su = np.asarray(R.sqd.uniquify_states(pack(bits), 2000))
    out['xsource'] = np.stack([np.asarray(R.sqd.get_xsource(xx, su))
                               for xx in ham.x]).astype(np.int32)
    return out


def even_y_pauli_sum(n, m, rng):
    """Random Pauli sum whose terms carry an even number of Y (real phased coefficients, so the
    reference's real-valued solve applies)."""
    x, z, c = W.random_pauli_sum(n, m, rng)
    ny = np.array([bin(int(a & b)).count('1') for a, b in zip(x, z)])
    keep = ny % 2 == 0
    return x[keep], z[keep], c[keep]


def real_solves(R, rec):
    out = {}
    cases = []
    # JW, 6 orbitals (12 qubits), 20 x 20 product subspace, shuffled input with repeats and
    # states_size above the unique count (fill rows)
    wl = W.jw_workload('jw6', 6, 3, 20, 20, 11)
    rng = np.random.default_rng(505)
    samples = np.concatenate([wl.states, rng.choice(wl.states, size=50)])
    rng.shuffle(samples)
    cases.append(('jw6', wl.x, wl.z, wl.coeffs, 12, samples, 470))
    # random even-Y Pauli sum on 12 qubits, 500 weight-6 strings
    x, z, c = even_y_pauli_sum(12, 200, rng)
    cases.append(('evy12', x, z, c, 12, W.weight_subspace(12, 6, 500, rng), None))
    # JW, 8 orbitals (16 qubits), 40 x 36 product subspace
    wl8 = W.jw_workload('jw8', 8, 3, 40, 36, 12)
    cases.append(('jw8', wl8.x, wl8.z, wl8.coeffs, 16, wl8.states, None))
    for tag, x, z, c, n, samples, size in cases:
        labels = W.labels_from_xz(x, z, n)
        bits = bits_of(samples, n)
        d = size if size is not None else bits.shape[0]
        probes = np.stack([rng.standard_normal(d) + 1j * rng.standard_normal(d)])
        t0 = time.time()
        e, vec, basis = run_sqd_capture(R, rec, (labels, list(c)), bits, size, (1, 0), probes,
                                        solve=True)
        out.update({f'{tag}_labels': labels_array(labels), f'{tag}_coeffs': c,
                    f'{tag}_bits': bits, f'{tag}_size': np.array(-1 if size is None else size),
                    f'{tag}_energy': np.array(e), f'{tag}_eigvec': np.asarray(vec),
                    f'{tag}_basis': np.asarray(basis), f'{tag}_niter': np.array(rec.niter),
                    f'{tag}_vinit': np.array(rec.vinit), f'{tag}_probes': probes,
                    f'{tag}_hv': rec.hv})
        print(f'  {tag}: E0 {e:.12f}, {rec.niter} iterations, {time.time() - t0:.1f} s',
              flush=True)
    # the jw6 solve capped at 12 iterations (iteration-by-iteration parity)
    tag, x, z, c, n, samples, size = cases[0]
    labels = W.labels_from_xz(x, z, n)
    e, vec, _ = run_sqd_capture(R, rec, (labels, list(c)), bits_of(samples, n), size, (1, 0),
                                probes[:0], solve=True, maxiter=12)
    out['jw6_cap12_energy'] = np.array(e)
    out['jw6_cap12_niter'] = np.array(rec.niter)
    out['jw6_cap12_eigvec'] = np.asarray(vec)
    return out


def dense_locg(R):
    rng = np.random.default_rng(606)
    a = rng.standard_normal((80, 80))
    mat = (a + a.T) / 2
    gl = R.ground_locg.ground_locg
    out = {'mat': mat}
    e0, v0, n0 = gl(mat, 0)
    out.update(e_int=np.array(e0), v_int=np.asarray(v0), n_int=np.array(n0))
    x0 = rng.standard_normal(80)
    out['xinit'] = x0
    e1, v1, n1 = gl(mat, x0, tol=1e-12)
    out.update(e_vec=np.array(e1), v_vec=np.asarray(v1), n_vec=np.array(n1))
    e2, v2, n2 = gl(mat, x0, orth=(np.asarray(v1),), tol=1e-12)
    out.update(e_orth=np.array(e2), v_orth=np.asarray(v2), n_orth=np.array(n2))
    return out


def eig_small(R):
    rng = np.random.default_rng(707)
    mats2, mats3 = [], []
    for _ in range(16):
        a = rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))
        mats2.append((a + a.conj().T) / 2)
        b = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
        mats3.append((b + b.conj().T) / 2)
    for _ in range(4):                             # real symmetric
        b = rng.standard_normal((3, 3))
        mats3.append((b + b.T) / 2 + 0j)

    def rotated(vals):
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3)))
        return (q * np.asarray(vals)) @ q.conj().T

    # lowest pair (near-)degenerate, upper pair (near-)degenerate, well separated
    for vals in ((1.0, 1.0 + 1e-9, 3.0), (1.0, 1.0 + 1e-6, 3.0), (-2.0, 0.5, 0.5 + 1e-7),
                 (-2.0, 0.5, 0.5), (0.1, 0.2, 0.3)):
        mats3.append(rotated(vals))
    mats2 = np.array(mats2)
    mats3 = np.array(mats3)
    e2 = [R.ground_locg.eigenpair_2x2(m) for m in mats2]
    e3 = [R.ground_locg.eigenpair_3x3(m) for m in mats3]
    return {'mats2': mats2, 'val2': np.array([float(v) for v, _ in e2]),
            'vec2': np.array([np.asarray(u) for _, u in e2]),
            'mats3': mats3, 'val3': np.array([float(v) for v, _ in e3]),
            'vec3': np.array([np.asarray(u) for _, u in e3])}


def main(reference_root='/root/reference'):
    R = reference_loader.load(reference_root)
    rec = Recorder(R)
    jobs = (('reference_paulis', lambda: paulis_case(R)),
            ('reference_subspace', lambda: subspace_case(R, rec)),
            ('reference_c1', lambda: c1_case(R, rec)),
            ('reference_solves', lambda: real_solves(R, rec)),
            ('reference_dense_locg', lambda: dense_locg(R)),
            ('reference_eig_small', lambda: eig_small(R)))
    for name, job in jobs:
        t0 = time.time()
        data = job()
        np.savez_compressed(os.path.join(HERE, name + '.npz'), **data)
        print(f'{name}: {len(data)} arrays, {time.time() - t0:.1f} s', flush=True)


if __name__ == '__main__':
    main(*sys.argv[1:2])
