"""The CPU oracle against fixtures written by the reference's OWN code (``reference_*.npz``, made
by ``tests/golden/make_reference_golden.py``, which runs the unmodified rqutils modules through
a NumPy stand-in for JAX).  Integer and index outputs must match bit for bit; floating-point
outputs within the tolerances below (the stand-in sums in NumPy's order, the oracle in its own,
XLA in a third: reductions differ in the last bits).
"""
import os
import warnings

import numpy as np
import pytest

from oracle import symplectic as OS, sqd as OQ, ground_locg as OL

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
SUM_RTOL = 1e-13          # same terms summed in another order
ENERGY_RTOL = 1e-12       # converged LOCG energies, same iteration
VEC_ATOL = 1e-8           # eigenvectors (phase-aligned)


def load(name):
    d = np.load(os.path.join(GOLDEN, name + '.npz'))
    return {k: d[k] for k in d.files}


def labels(arr):
    return [s.decode() for s in arr]


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


def aligned(v, ref):
    """``v`` times the unit phase that best aligns it with ``ref``."""
    ip = np.vdot(v, ref)
    return v * (ip / abs(ip))


# ----------------------------------------------------------------------------- Pauli tables
@pytest.mark.parametrize('tag,coeff_key,kw', [
    ('real_pad', 'coeffs', dict(add_padding=True)),
    ('real_nopad', 'coeffs', dict()),
    ('cplx_nopad', 'coeffs_complex', dict()),
    ('cplx_forcereal_pad', 'coeffs_complex', dict(force_real=True, add_padding=True))])
def test_from_paulisum_matches_reference(tag, coeff_key, kw):
    g = load('reference_paulis')
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter('always')
        h = OS.from_paulisum((labels(g['labels']), list(g[coeff_key])), **kw)
    np.testing.assert_array_equal(h.x, g[f'{tag}_x'])
    np.testing.assert_array_equal(h.z, g[f'{tag}_z'])
    assert h.c.dtype == g[f'{tag}_c'].dtype
    np.testing.assert_array_equal(h.c, g[f'{tag}_c'])
    warned = any('imaginary' in str(w.message) for w in caught)
    assert warned == bool(g[f'{tag}_warned'])


# ----------------------------------------------------------------------------- subspace
@pytest.mark.parametrize('tag,size', [('plus', 200), ('exact', 180), ('minus', 170),
                                      ('all', 240)])
def test_uniquify_states_matches_reference(tag, size):
    g = load('reference_subspace')
    su, idx = OQ.uniquify_states(g['packed'], size, return_indices=True)
    np.testing.assert_array_equal(su, g[f'uniq_{tag}'])
    np.testing.assert_array_equal(idx, g[f'uniq_{tag}_idx'])


def test_packing_matches_reference_rows():
    g = load('reference_subspace')
    np.testing.assert_array_equal(OQ.pack_states(g['bits']), g['packed'])


def test_get_xsource_and_diagonal_match_reference():
    g = load('reference_subspace')
    su = OQ.uniquify_states(g['packed'], 200)
    for j, x in enumerate(g['x']):
        np.testing.assert_array_equal(OQ.get_xsource(x, su), g['xsource'][j])
        np.testing.assert_array_equal(OQ.get_diagonal(g['z'][j], g['c'][j], su),
                                      g['diagonal'][j])
    usp = OQ.pack_states(g['unsorted_bits'])
    for j, x in enumerate(g['x']):
        np.testing.assert_array_equal(OQ.get_xsource_unsorted(x, usp),
                                      g['xsource_unsorted'][j])


@pytest.mark.parametrize('cache', ['10', '12', '00', '02'])
def test_assembled_matvec_and_vinit_match_reference(cache):
    """run_sqd's matvec for each cache strategy (fill rows included) and its start index."""
    g = load('reference_subspace')
    ham = OS.from_paulisum((labels(g['labels']), list(g['coeffs'])), force_real=True,
                           add_padding=True)
    su = OQ.uniquify_states(OQ.pack_states(g['bits']), 260)
    xs = np.stack([OQ.get_xsource(x, su) for x in ham.x])
    for p, hv in zip(g['probes'], g[f'hv_{cache}']):
        assert rel(OQ.apply_h_x_cached(p, xs, ham.z, ham.c, su), hv) < SUM_RTOL
    assert OQ.vinit_index(ham, su) == int(g[f'vinit_{cache}'])


def test_c1_connectivity_matvec_and_vinit_match_reference():
    from rqutils_b200 import workloads as W
    g = load('reference_c1')
    wl = W.c1(0)
    bits = OQ.u64_to_states(wl.states, 16)
    ham = OS.from_paulisum((wl.labels, list(wl.coeffs)), force_real=True, add_padding=True)
    su = OQ.uniquify_states(OQ.pack_states(bits), 2000)
    xs = np.stack([OQ.get_xsource(x, su) for x in ham.x])
    np.testing.assert_array_equal(xs, g['xsource'])
    for cache in ('10', '12'):
        assert rel(OQ.apply_h_x_cached(g['probes'][0], xs, ham.z, ham.c, su),
                   g[f'hv_{cache}'][0]) < SUM_RTOL
        assert OQ.vinit_index(ham, su) == int(g[f'vinit_{cache}'])


# ----------------------------------------------------------------------------- solves
@pytest.mark.parametrize('tag', ['jw6', 'evy12', 'jw8'])
def test_sqd_solve_matches_reference(tag):
    g = load('reference_solves')
    size = int(g[f'{tag}_size'])
    size = None if size < 0 else size
    lab, c, bits = labels(g[f'{tag}_labels']), g[f'{tag}_coeffs'], g[f'{tag}_bits']
    e, vec, basis = OQ.sqd((lab, list(c)), bits, states_size=size)
    np.testing.assert_array_equal(basis, g[f'{tag}_basis'])
    assert abs(e - float(g[f'{tag}_energy'])) <= ENERGY_RTOL * abs(e)
    assert np.abs(aligned(vec, g[f'{tag}_eigvec']) - g[f'{tag}_eigvec']).max() < VEC_ATOL
    ham = OS.from_paulisum((lab, list(c)), force_real=True, add_padding=True)
    su = OQ.uniquify_states(OQ.pack_states(bits), size or bits.shape[0])
    assert OQ.vinit_index(ham, su) == int(g[f'{tag}_vinit'])
    *_, niter = OQ.run_sqd(ham, OQ.pack_states(bits), size or bits.shape[0])
    assert abs(niter - int(g[f'{tag}_niter'])) <= 2


def test_capped_iteration_count_matches_reference():
    """maxiter=12: the reference stops after exactly 12 body iterations; the energy there
    (unconverged) pins the iteration itself, not just its fixed point."""
    g = load('reference_solves')
    lab, c, bits = labels(g['jw6_labels']), g['jw6_coeffs'], g['jw6_bits']
    ham = OS.from_paulisum((lab, list(c)), force_real=True, add_padding=True)
    opts = OQ.SQDOptions(locg_maxiter=12)
    e, vec, _, _, niter = OQ.run_sqd(ham, OQ.pack_states(bits), int(g['jw6_size']), opts)
    assert niter == int(g['jw6_cap12_niter']) == 12
    assert abs(e - float(g['jw6_cap12_energy'])) <= 1e-12 * abs(e)


def test_dense_ground_locg_matches_reference():
    g = load('reference_dense_locg')
    mat = g['mat']
    e, v, n = OL.ground_locg(mat, 0)
    assert abs(e - float(g['e_int'])) <= ENERGY_RTOL * abs(e) and abs(n - int(g['n_int'])) <= 2
    e, v, n = OL.ground_locg(mat, g['xinit'], tol=1e-12)
    assert abs(e - float(g['e_vec'])) <= ENERGY_RTOL * abs(e) and abs(n - int(g['n_vec'])) <= 2
    e2, v2, n2 = OL.ground_locg(mat, g['xinit'], orth=(g['v_vec'],), tol=1e-12)
    assert abs(e2 - float(g['e_orth'])) <= 1e-10 * abs(e2)


def test_small_eigenpairs_match_reference():
    g = load('reference_eig_small')
    for m, val, vec in zip(g['mats2'], g['val2'], g['vec2']):
        e, u = OL.eigenpair_2x2(m)
        assert abs(e - val) <= 1e-13 * max(1.0, abs(val))
        np.testing.assert_allclose(u, vec, rtol=0, atol=1e-12)
    for m, val, vec in zip(g['mats3'], g['val3'], g['vec3']):
        e, u = OL.eigenpair_3x3(m)
        assert abs(e - val) <= 1e-13 * max(1.0, abs(val))
        if np.all(np.isfinite(vec)):
            np.testing.assert_allclose(u, vec, rtol=0, atol=1e-9)
