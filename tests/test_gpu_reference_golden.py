"""The CUDA path against outputs of the reference's OWN code (``tests/golden/reference_*.npz``,
written by ``tests/golden/make_reference_golden.py`` from the unmodified rqutils modules run
through a NumPy stand-in for JAX).

Bit-exact: Pauli tables, packed-row ``uniquify_states`` (rows and indices), ``get_xsource``
(sorted input with fill rows, unsorted input), group diagonals (same term order), start
indices, the basis of every solve.  Floating point: matvecs 1e-13 of the largest entry
(association order differs); energies 1e-10 relative (the reference iterates to its own
N-scaled stopping test, so converged energies agree to far below that); the 12-iteration capped
solve 1e-10 (same iteration, different reduction order); iteration counts within 2; small
eigenpairs 1e-12.
"""
import ctypes
import os
import warnings

import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import _lib, workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
MATVEC_RTOL = 1e-13
ENERGY_RTOL = 1e-10


def load(name):
    d = np.load(os.path.join(GOLDEN, name + '.npz'))
    return {k: d[k] for k in d.files}


def labels(arr):
    return [s.decode() for s in arr]


def rel(a, b):
    return np.abs(np.asarray(a) - b).max() / max(np.abs(b).max(), 1e-300)


def host(t):
    return t.cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


@pytest.mark.parametrize('tag,coeff_key,kw', [
    ('real_pad', 'coeffs', dict(add_padding=True)),
    ('real_nopad', 'coeffs', dict()),
    ('cplx_nopad', 'coeffs_complex', dict()),
    ('cplx_forcereal_pad', 'coeffs_complex', dict(force_real=True, add_padding=True))])
def test_device_pauli_preprocessing_matches_reference(tag, coeff_key, kw):
    g = load('reference_paulis')
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter('always')
        ham = rq.PauliSumXZ.from_paulisum((labels(g['labels']), list(g[coeff_key])), **kw)
    np.testing.assert_array_equal(ham.x, g[f'{tag}_x'])
    np.testing.assert_array_equal(ham.z, g[f'{tag}_z'])
    assert ham.c.dtype == g[f'{tag}_c'].dtype
    np.testing.assert_array_equal(ham.c, g[f'{tag}_c'])
    assert any('imaginary' in str(w.message) for w in caught) == bool(g[f'{tag}_warned'])


@pytest.mark.parametrize('tag,size', [('plus', 200), ('exact', 180), ('minus', 170),
                                      ('all', 240)])
def test_packed_uniquify_matches_reference(tag, size):
    g = load('reference_subspace')
    su, idx = rq.uniquify_states(g['packed'], size, return_indices=True)
    np.testing.assert_array_equal(host(su), g[f'uniq_{tag}'])
    np.testing.assert_array_equal(host(idx), g[f'uniq_{tag}_idx'])


@pytest.mark.parametrize('lookup', ['hash', 'bsearch'])
def test_xsource_sorted_and_unsorted_match_reference(lookup):
    g = load('reference_subspace')
    su = g['uniq_plus']
    for j, x in enumerate(g['x']):
        got = rq.get_xsource(x, su, lookup=lookup)
        np.testing.assert_array_equal(host(got), g['xsource'][j], err_msg=f'group {j}')
    usp = np.packbits(np.pad(g['unsorted_bits'], ((0, 0), (1, 0))), axis=1)
    for j, x in enumerate(g['x']):
        got = rq.get_xsource(x, usp, sorted_input=False, lookup=lookup)
        np.testing.assert_array_equal(host(got), g['xsource_unsorted'][j])


@pytest.mark.parametrize('cache', [(1, 0), (1, 2), (0, 0), (0, 2)])
def test_matvec_diagonals_and_vinit_match_reference(cache):
    """The 10-qubit complex case with 180 unique rows and 80 fill rows."""
    g = load('reference_subspace')
    ham = rq.PauliSumXZ.from_paulisum((labels(g['labels']), list(g['coeffs'])),
                                      force_real=True, add_padding=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_bits(g['bits'], 260), cache_strategy=cache)
    key = f'{cache[0]}{cache[1]}'
    for p, hv in zip(g['probes'], g[f'hv_{key}']):
        assert rel(op.matvec(torch.as_tensor(p, device='cuda')).cpu().numpy(), hv) < MATVEC_RTOL
    assert op.vinit() == int(g[f'vinit_{key}'])
    if cache == (1, 0):
        op200 = rq.SQDOperator(ham, rq.Subspace.from_bits(g['bits'], 260))
        for j in range(g['diagonal'].shape[0]):
            d = op200.diagonal(j).cpu().numpy()[:180]
            np.testing.assert_array_equal(d, g['diagonal'][j][:180])


def test_c1_connectivity_matvec_and_vinit_match_reference():
    g = load('reference_c1')
    wl = W.c1(0)
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, 16, force_real=True, padded=True)
    space = rq.Subspace.from_u64(wl.states, 16)
    gx = ham.device_tables()[0].cpu().numpy().view(np.uint64)
    for j, x in enumerate(gx):
        np.testing.assert_array_equal(space.xsource(int(x)).cpu().numpy(), g['xsource'][j])
    for cache in ((1, 0), (1, 2)):
        op = rq.SQDOperator(ham, space, cache_strategy=cache)
        hv = op.matvec(torch.as_tensor(g['probes'][0], device='cuda')).cpu().numpy()
        assert rel(hv, g[f'hv_{cache[0]}{cache[1]}'][0]) < MATVEC_RTOL
        assert op.vinit() == int(g[f'vinit_{cache[0]}{cache[1]}'])


@pytest.mark.parametrize('tag', ['jw6', 'evy12', 'jw8'])
@pytest.mark.parametrize('mode', ['fp64', 'mixed'])
def test_sqd_solves_match_reference(tag, mode):
    g = load('reference_solves')
    size = int(g[f'{tag}_size'])
    size = None if size < 0 else size
    lab, c, bits = labels(g[f'{tag}_labels']), list(g[f'{tag}_coeffs']), g[f'{tag}_bits']
    if mode == 'fp64':
        e, vec, basis = rq.sqd((lab, c), bits, states_size=size)
        np.testing.assert_array_equal(basis, g[f'{tag}_basis'])
        ref = g[f'{tag}_eigvec']
        ip = np.vdot(vec, ref)
        assert np.abs(vec * (ip / abs(ip)) - ref).max() < 1e-7
    ham = rq.PauliSumXZ.from_paulisum((lab, c), force_real=True, add_padding=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_bits(bits, size))
    assert op.vinit() == int(g[f'{tag}_vinit'])
    hv = op.matvec(torch.as_tensor(g[f'{tag}_probes'][0], device='cuda')).cpu().numpy()
    assert rel(hv, g[f'{tag}_hv'][0]) < MATVEC_RTOL
    e, _, niter = rq.ground_locg(op, op.vinit(), mode=mode, vspace=(op.size, torch.float64))
    e_ref = float(g[f'{tag}_energy'])
    assert abs(e - e_ref) <= ENERGY_RTOL * abs(e_ref)
    if mode == 'fp64':
        assert abs(niter - int(g[f'{tag}_niter'])) <= 2


def test_capped_solve_matches_reference_iteration():
    g = load('reference_solves')
    lab, c, bits = labels(g['jw6_labels']), list(g['jw6_coeffs']), g['jw6_bits']
    ham = rq.PauliSumXZ.from_paulisum((lab, c), force_real=True, add_padding=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_bits(bits, int(g['jw6_size'])))
    for graph in (False, True):
        e, vec, niter = rq.ground_locg(op, op.vinit(), maxiter=12, use_graph=graph,
                                       vspace=(op.size, torch.float64))
        assert niter == int(g['jw6_cap12_niter']) == 12
        assert abs(e - float(g['jw6_cap12_energy'])) <= ENERGY_RTOL * abs(e)


def test_dense_ground_locg_matches_reference():
    g = load('reference_dense_locg')
    mat = torch.as_tensor(g['mat'], device='cuda')
    e, v, n = rq.ground_locg(mat, 0)
    assert abs(e - float(g['e_int'])) <= 1e-12 * abs(e) and abs(n - int(g['n_int'])) <= 2
    x0 = torch.as_tensor(g['xinit'], device='cuda')
    e, v, n = rq.ground_locg(mat, x0, tol=1e-12)
    assert abs(e - float(g['e_vec'])) <= 1e-12 * abs(e) and abs(n - int(g['n_vec'])) <= 2
    e2, _, _ = rq.ground_locg(mat, x0, orth=(torch.as_tensor(g['v_vec'], device='cuda'),),
                              tol=1e-12)
    assert abs(e2 - float(g['e_orth'])) <= 1e-10 * abs(e2)


def _device_eigenpairs(mats):
    count, dim = mats.shape[0], mats.shape[1]
    m = torch.as_tensor(np.ascontiguousarray(mats), device='cuda')
    vals = torch.empty(count, dtype=torch.float64, device='cuda')
    vecs = torch.empty((count, dim), dtype=torch.complex128, device='cuda')
    _lib.call('sqd_eigenpair_small', _lib.ptr(m), ctypes.c_int64(count), dim, _lib.ptr(vals),
              _lib.ptr(vecs), _lib.stream_ptr())
    return vals.cpu().numpy(), vecs.cpu().numpy()


def test_small_eigenpairs_match_reference_and_eigh():
    """eigenpair_2x2 / eigenpair_3x3 on random, degenerate and near-degenerate Hermitian
    matrices.  Cardano's method loses about half the digits when two eigenvalues nearly meet,
    so the bar depends on the smallest gap g of the spectrum (scale s = max |eigenvalue|):
    g > 1e-3 s: value within 1e-12 s of the reference's and of numpy.linalg.eigh, vector within
    1e-9 of the reference's; closer eigenvalues: value within 1e-7 s of eigh (the reference's
    own value may be NaN there: its square roots take arguments that rounding can push below
    zero, which the device code clamps at 0)."""
    g = load('reference_eig_small')
    for key in ('2', '3'):
        mats, vals_ref, vecs_ref = g['mats' + key], g['val' + key], g['vec' + key]
        vals, vecs = _device_eigenpairs(mats)
        assert np.isfinite(vals).all()
        for m, val, vec, vr, ur in zip(mats, vals, vecs, vals_ref, vecs_ref):
            w = np.linalg.eigvalsh(m)
            scale = max(1.0, np.abs(w).max())
            gap = np.diff(w).min()
            if gap > 1e-3 * scale:
                assert abs(val - vr) <= 1e-12 * scale
                assert abs(val - w[0]) <= 1e-12 * scale
                np.testing.assert_allclose(vec, ur, rtol=0, atol=1e-9)
                assert np.linalg.norm(m @ vec - val * vec) <= 1e-10 * scale
            else:
                assert abs(val - w[0]) <= 1e-7 * scale


def test_small_eigenpairs_reject_bad_dimensions():
    st = _lib.load().sqd_eigenpair_small(None, 1, 4, None, None, None)
    assert st == _lib.SQD_ERR_INVALID


def test_debug_log_level_records_and_prints_every_iteration(capsys):
    """log_level=DEBUG: the reference's per-iteration lines (ground_locg.py:330-331, 377-378),
    from the record the device solver writes; the residual sequence follows the oracle's
    iteration of the same algorithm (FP64, another summation order) step by step."""
    import logging
    from oracle import symplectic as OS, sqd as OQ, ground_locg as OL
    g = load('reference_solves')
    lab, c, bits = labels(g['jw6_labels']), list(g['jw6_coeffs']), g['jw6_bits']
    size = int(g['jw6_size'])
    ham = rq.PauliSumXZ.from_paulisum((lab, c), force_real=True, add_padding=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_bits(bits, size))
    capsys.readouterr()
    e, _, niter = rq.ground_locg(op, op.vinit(), vspace=(op.size, torch.float64),
                                 log_level=logging.DEBUG)
    out = capsys.readouterr().out
    hist = rq.ground_locg.last_history
    assert out.count('LOCG iteration') == niter == hist.shape[0]
    assert (hist[:, 0] == 0).all() and (hist[:, 1] == np.arange(1, niter + 1)).all()
    assert hist[-1, 5] == 1 and (hist[:-1, 5] == 0).all() and hist[-1, 2] == e
    oham = OS.from_paulisum((lab, c), force_real=True, add_padding=True)
    su = OQ.uniquify_states(OQ.pack_states(bits), size)
    xs = np.stack([OQ.get_xsource(x, su) for x in oham.x])
    *_, hist_o = OL.ground_locg(lambda v: OQ.apply_h_x_cached(v, xs, oham.z, oham.c, su),
                                OQ.vinit_index(oham, su), vspace=(size, np.float64),
                                return_history=True)
    k = min(30, niter)
    np.testing.assert_allclose(hist[:k, 3], hist_o[:k], rtol=1e-6)
    # mixed precision: FP32 sweeps first (phase 1), then FP64 iterations (phase 0)
    e_m, _, niter_m = rq.ground_locg(op, op.vinit(), vspace=(op.size, torch.float64),
                                     mode='mixed', log_level=logging.DEBUG)
    hist_m = rq.ground_locg.last_history
    phases = hist_m[:, 0]
    assert hist_m.shape[0] == niter_m and phases[0] == 1
    assert (np.diff(phases) <= 0).all()          # 1 ... 1 0 ... 0
    assert hist_m[-1, 5] == 1 and abs(hist_m[-1, 2] - e_m) == 0
    # no record without the debug level
    capsys.readouterr()
    rq.ground_locg(op, op.vinit(), vspace=(op.size, torch.float64))
    assert 'LOCG iteration' not in capsys.readouterr().out
