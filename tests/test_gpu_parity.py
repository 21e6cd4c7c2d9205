"""GPU parity against the CPU oracle on small seeded inputs (bit-exact for integer/index work,
tolerances written per test for floating point)."""
import os

import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import workloads as W
from oracle import symplectic as OS, sqd as OQ, dense as OD, ground_locg as OL

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')

# Tolerances: FP64 matvec vs the oracle's sequential sums (different association order)
MATVEC_RTOL = 1e-13
# FP32 compensated matvec vs FP64 oracle
MATVEC32_RTOL = 2e-6
ENERGY_RTOL = 1e-8


def golden(name):
    d = np.load(os.path.join(GOLDEN, name + '.npz'))
    return {k: d[k] for k in d.files}


def labels_of(g):
    return [s.decode() for s in g['labels']]


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


# ----------------------------------------------------------------------------- Pauli tables
@pytest.mark.parametrize('cplx', [False, True])
def test_pauli_preprocessing_matches_reference_layout(cplx):
    g = golden('paulis_small')
    labels = labels_of(g)
    coeffs = g['coeffs_complex'] if cplx else g['coeffs']
    ham = rq.PauliSumXZ.from_paulisum((labels, list(coeffs)), add_padding=not cplx)
    x, z, c = (g['xc'], g['zc'], g['cc']) if cplx else (g['x'], g['z'], g['c'])
    np.testing.assert_array_equal(ham.x, x)
    np.testing.assert_array_equal(ham.z, z)
    assert ham.c.dtype == c.dtype
    # merged duplicates are sums of two values: exact; others copied with an exact phase
    np.testing.assert_array_equal(ham.c, c)


def test_force_real_warns_and_drops_imaginary_parts():
    g = golden('paulis_small')
    with pytest.warns(UserWarning, match='imaginary'):
        ham = rq.PauliSumXZ.from_paulisum((labels_of(g), list(g['coeffs_complex'])),
                                          force_real=True, add_padding=True)
    ref = OS.from_paulisum((labels_of(g), list(g['coeffs_complex'])), force_real=True,
                           add_padding=True)
    np.testing.assert_array_equal(ham.c, ref.c)


def test_pauli_roundtrip_from_reference_arrays():
    g = golden('paulis_small')
    ham = rq.PauliSumXZ(g['x'], g['z'], g['c'], 10)
    np.testing.assert_array_equal(ham.x, g['x'])
    np.testing.assert_array_equal(ham.z, g['z'])
    np.testing.assert_allclose(ham.c, g['c'], rtol=0, atol=0)


# ----------------------------------------------------------------------------- subspace
def test_uniquify_and_xsource_bit_exact():
    g = golden('sqd_small')
    size = int(g['states_size'])
    space = rq.Subspace.from_bits(g['states'], size)
    assert space.n_unique == 150 and space.states_size == size
    np.testing.assert_array_equal(space.states().cpu().numpy().view(np.uint64), g['states_u64'])
    ham = OS.from_paulisum((labels_of(g), list(g['coeffs'])), force_real=True, add_padding=True)
    xm = [int(v) for v in OQ.packed_to_u64(ham.x, 10)]
    for lookup in ('hash', 'bsearch'):
        for j, x in enumerate(xm):
            got = space.xsource(x, lookup).cpu().numpy()
            np.testing.assert_array_equal(got, g['xsources'][j], err_msg=f'group {j} {lookup}')


def test_pack_states_matches_reference_order():
    rng = np.random.default_rng(5)
    bits = rng.integers(0, 2, size=(3000, 37)).astype(np.uint8)
    space = rq.Subspace.from_bits(bits)
    ref = np.unique(OQ.states_to_u64(bits))
    np.testing.assert_array_equal(space.states().cpu().numpy().view(np.uint64), ref)
    np.testing.assert_array_equal(space.states_bits(), np.unique(bits, axis=0))


# ----------------------------------------------------------------------------- operator
@pytest.mark.parametrize('cache', [(1, 0), (1, 1), (1, 2), (0, 0), (0, 2)])
@pytest.mark.parametrize('lookup', ['hash', 'bsearch'])
def test_matvec_matches_oracle_with_fill_slots(cache, lookup):
    g = golden('sqd_small')
    size = int(g['states_size'])
    ham = rq.PauliSumXZ.from_paulisum((labels_of(g), list(g['coeffs'])), force_real=True,
                                      add_padding=True)
    space = rq.Subspace.from_bits(g['states'], size)
    op = rq.SQDOperator(ham, space, cache_strategy=cache, lookup=lookup)
    v = torch.as_tensor(g['v'], device='cuda')
    hv = op.matvec(v).cpu().numpy()
    assert rel(hv, g['hv']) < MATVEC_RTOL
    # fill-in slot with a nonzero amplitude: the reference maps the last slot to the first
    v2 = v.clone()
    v2[150] = 0.7 - 0.2j
    d0 = OQ.get_diagonal(OS.from_paulisum((labels_of(g), list(g['coeffs'])), force_real=True,
                                          add_padding=True).z[0],
                         OS.from_paulisum((labels_of(g), list(g['coeffs'])), force_real=True,
                                          add_padding=True).c[0],
                         np.full((size, 2), 255, dtype=np.uint8))
    hv2 = op.matvec(v2).cpu().numpy()
    assert abs(hv2[size - 1] - d0[0] * (0.7 - 0.2j)) < 1e-12
    np.testing.assert_allclose(hv2[:150], hv[:150], rtol=0, atol=1e-13)


@pytest.mark.parametrize('cache', [(1, 0), (1, 2), (0, 0)])
def test_matvec_fp32_compensated(cache):
    g = golden('sqd_small')
    size = int(g['states_size'])
    ham = rq.PauliSumXZ.from_paulisum((labels_of(g), list(g['coeffs'])), force_real=True,
                                      add_padding=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_bits(g['states'], size), cache_strategy=cache)
    v = torch.as_tensor(g['v'], device='cuda')
    hv32 = op.matvec(v.to(torch.complex64)).cpu().numpy()
    ref = OQ.apply_h_x_cached(g['v'].astype(np.complex64).astype(np.complex128),
                              g['xsources'],
                              *OS.from_paulisum((labels_of(g), list(g['coeffs'])),
                                                force_real=True, add_padding=True).arrays[1:],
                              OQ.uniquify_states(OQ.pack_states(g['states']), size))
    assert rel(hv32, ref) < MATVEC32_RTOL


@pytest.mark.parametrize('lanes', [1, 2, 4, 8, 16, 32])
def test_matvec_every_schedule(lanes):
    wl = W.c1(0)
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, 16, force_real=True, padded=True)
    space = rq.Subspace.from_u64(wl.states, 16)
    oham = OS.from_paulisum((wl.labels, list(wl.coeffs)), force_real=True, add_padding=True)
    sp = OQ.pack_states(OQ.u64_to_states(wl.states, 16))
    xs = np.stack([OQ.get_xsource(x, sp) for x in oham.x])
    v = wl.start_vector()
    ref = OQ.apply_h_x_cached(v, xs, oham.z, oham.c, sp)
    for cache in ((1, 0), (1, 2)):
        op = rq.SQDOperator(ham, space, cache_strategy=cache, lanes_per_row=lanes)
        hv = op.matvec(torch.as_tensor(v, device='cuda')).cpu().numpy()
        assert rel(hv, ref) < MATVEC_RTOL


def test_diagonal_vinit_and_csr():
    g = golden('sqd_small')
    size = int(g['states_size'])
    ham = rq.PauliSumXZ.from_paulisum((labels_of(g), list(g['coeffs'])), force_real=True,
                                      add_padding=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_bits(g['states'], size))
    # group-0 diagonal: same term order as the reference -> bit-exact
    np.testing.assert_array_equal(op.diagonal(0).cpu().numpy(), g['diag0'])
    assert op.vinit() == int(g['vinit'])
    h = rq.hproj((labels_of(g), list(g['coeffs'])), g['states'])
    dense = OD.projected_matrix(labels_of(g), g['coeffs'], g['states_u64'])
    np.testing.assert_allclose(h.toarray(), dense, rtol=0, atol=1e-12)


# ----------------------------------------------------------------------------- LOCG
def test_locg_matches_oracle_iteration_by_iteration():
    g = golden('sqd_small')
    size = int(g['states_size'])
    ham = rq.PauliSumXZ.from_paulisum((labels_of(g), list(g['coeffs'])), force_real=True,
                                      add_padding=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_bits(g['states'], size))
    for graph in (False, True):
        e, vec, niter = rq.ground_locg(op, int(g['vinit']), tol=1e-12, use_graph=graph)
        assert abs(e - float(g['eig_locg'])) <= 1e-12 * abs(float(g['eig_locg']))
        assert abs(niter - int(g['niter'])) <= 2
        assert abs(e - float(g['eig_dense'])) <= ENERGY_RTOL * abs(float(g['eig_dense']))
        assert torch.all(vec[150:] == 0)


def test_sqd_notebook_recipe_matches_dense():
    g = golden('notebook_small')
    e = rq.sqd((labels_of(g), list(g['coeffs'])), g['states'], options={'locg_tol': 1e-12,
                                                                      'return_eigvec': False})
    assert abs(e - float(g['eig_dense'])) <= ENERGY_RTOL * abs(float(g['eig_dense']))
    assert abs(e - float(g['eig_oracle'])) <= 1e-10 * abs(float(g['eig_dense']))


def test_sqd_c1_against_dense_eigh():
    wl = W.c1(0)
    bits = OQ.u64_to_states(wl.states, 16)
    e, vec, basis = rq.sqd((wl.labels, list(wl.coeffs)), bits, options={'locg_tol': 1e-10})
    h = OD.projected_matrix(wl.labels, wl.coeffs, OQ.states_to_u64(basis))
    w, u = np.linalg.eigh(h)
    assert abs(e - w[0]) <= ENERGY_RTOL * abs(w[0])
    assert abs(abs(np.vdot(u[:, 0], vec)) - 1) < 1e-6


def test_locg_c1_complex_start_vector():
    wl = W.c1(0)
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, 16, force_real=True, padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(wl.states, 16))
    x0 = torch.as_tensor(wl.start_vector(np.complex128), device='cuda')
    e, vec, it = rq.ground_locg(op, x0, tol=1e-10)
    assert vec.dtype == torch.complex128
    h = OD.projected_matrix(wl.labels, wl.coeffs, wl.states)
    e0 = np.linalg.eigvalsh(h)[0]
    assert abs(e - e0) <= ENERGY_RTOL * abs(e0)


def test_ground_locg_callable_dense_and_orth():
    rng = np.random.default_rng(2)
    a = rng.standard_normal((80, 80)) + 1j * rng.standard_normal((80, 80))
    h = a + a.conj().T
    w, u = np.linalg.eigh(h)
    ht = torch.as_tensor(h, device='cuda')
    e, v, it = rq.ground_locg(ht, 0, tol=1e-12)
    eo, vo, ito = OL.ground_locg(h, 0, tol=1e-12)
    assert abs(e - w[0]) < 1e-9 * abs(w[0])
    assert abs(e - eo) < 1e-11 * abs(w[0]) and abs(it - ito) <= 2
    e2, _, _ = rq.ground_locg(lambda x, s: s * (ht @ x), 3, args=(2.0,), tol=1e-12,
                              vspace=(80, np.complex128))
    assert abs(e2 - 2 * w[0]) < 1e-9 * abs(w[0])
    e1, v1, _ = rq.ground_locg(ht, 5, orth=(torch.as_tensor(u[:, 0], device='cuda'),),
                               tol=1e-12)
    assert abs(e1 - w[1]) < 1e-8 * abs(w[1])


def test_ground_locg_vspace_required_for_callable():
    with pytest.raises(ValueError, match='vspace'):
        rq.ground_locg(lambda x: x, 0)


def test_mixed_precision_energy_matches_fp64():
    wl = W.c2_small(0, 96, 80)
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, 32, force_real=True, padded=True)
    for cache in ((1, 0), (1, 2)):
        op = rq.SQDOperator(ham, rq.Subspace.from_u64(wl.states, 32), cache_strategy=cache)
        v0 = op.vinit()
        e64, _, _ = rq.ground_locg(op, v0, tol=1e-10)
        em, _, _ = rq.ground_locg(op, v0, tol=1e-10, mode='mixed')
        assert abs(em - e64) <= ENERGY_RTOL * abs(e64)


def test_full_space_matmul_matches_oracle():
    rng = np.random.default_rng(8)
    x, z, c = W.random_pauli_sum(9, 40, rng)
    labels = W.labels_from_xz(x, z, 9)
    ham = rq.PauliSumXZ.from_paulisum((labels, list(c)))
    v = rng.standard_normal((512, 2)) + 1j * rng.standard_normal((512, 2))
    got = ham.matmul(torch.as_tensor(v, device='cuda')).cpu().numpy()
    ref = OS.matmul(OS.from_paulisum((labels, list(c))), v)
    assert rel(got, ref) < MATVEC_RTOL


def test_gradient_terms_match_hellmann_feynman_oracle():
    wl = W.c1(0)
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, 16, force_real=True, padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(wl.states, 16))
    rng = np.random.default_rng(3)
    v = rng.standard_normal(2000) + 1j * rng.standard_normal(2000)
    g = op.grad_terms(torch.as_tensor(v, device='cuda'), torch.as_tensor(v, device='cuda'))
    gx, gs, tz, tc, _ = (t.cpu().numpy() for t in ham.device_tables())
    gx, tz = gx.view(np.uint64), tz.view(np.uint64)
    # Hellmann-Feynman restated: Re <v| (-i)^{|x&z|} (-1)^{|s&z|} |v[src]>  per merged term
    s = wl.states
    pos = {int(val): k for k, val in enumerate(s)}
    ref = np.zeros(tz.shape[0])
    for j in range(gx.shape[0]):
        src = np.array([pos.get(int(val ^ gx[j]), -1) for val in s])
        ok = src >= 0
        w = np.conj(v[ok]) * v[src[ok]]
        for t in range(gs[j], gs[j + 1]):
            ph = (-1j) ** (int(np.bitwise_count(gx[j] & tz[t])) & 3)
            sign = 1. - 2. * (np.bitwise_count(s[ok] & tz[t]) & 1)
            ref[t] = np.real(ph * np.sum(sign * w))
    np.testing.assert_allclose(g.cpu().numpy(), ref, rtol=1e-10, atol=1e-9)
    # autograd-style check of one coordinate: d<v|H|v>/d alpha_t = g_t
    assert np.isfinite(ref).all()


def test_exact_eigenvector_start_returns_exact_pair():
    # Diagonal Hamiltonian: the one-hot vinit is an exact eigenvector (r = 0 after iteration 0).
    labels = ['ZIII', 'IZZI', 'IIZZ', 'ZIIZ']
    coeffs = [0.7, -1.1, 0.4, -0.3]
    states = OQ.u64_to_states(np.arange(16, dtype=np.uint64), 4)
    e, vec, basis = rq.sqd((labels, coeffs), states)
    dense = OD.projected_matrix(labels, coeffs, np.arange(16))
    assert np.isfinite(e) and abs(e - np.linalg.eigvalsh(dense)[0]) < 1e-14
    assert np.isfinite(vec).all()


def test_duplicate_and_unsorted_inputs_with_fill_slots():
    rng = np.random.default_rng(12)
    x, z, c = W.random_pauli_sum(9, 50, rng)
    labels = W.labels_from_xz(x, z, 9)
    base = W.weight_subspace(9, 4, 90, rng)
    sample = np.concatenate([base, base[:30], base[::-1]])
    bits = OQ.u64_to_states(sample, 9)
    size = bits.shape[0] + 5
    e, vec, basis = rq.sqd((labels, list(c)), bits, states_size=size,
                           options={'locg_tol': 1e-13})
    eo, veco, basiso = OQ.sqd((labels, list(c)), bits, states_size=size,
                              options={'locg_tol': 1e-13})
    assert (basis == basiso).all() and basis.shape[0] == 90
    assert abs(e - eo) <= 1e-10 * abs(eo)
    assert abs(abs(np.vdot(vec, veco)) - 1) < 1e-8


def test_sqd_reference_layout_pauli_input():
    g = golden('sqd_small')
    ref = OS.from_paulisum((labels_of(g), list(g['coeffs'])), force_real=True, add_padding=True)
    ham = rq.PauliSumXZ(ref.x, ref.z, ref.c, 10)
    e = rq.sqd(ham, g['states'], states_size=int(g['states_size']),
               options={'locg_tol': 1e-12, 'return_eigvec': False})
    assert abs(e - float(g['eig_dense'])) <= ENERGY_RTOL * abs(float(g['eig_dense']))


def test_invalid_inputs_raise_value_error():
    with pytest.raises(ValueError):
        rq.PauliSumXZ.from_xz(np.array([1], dtype=np.uint64), np.array([0], dtype=np.uint64),
                              np.array([0.0]), 4)       # every coefficient is zero
    with pytest.raises(ValueError):
        rq.Subspace.from_u64(np.array([1 << 9], dtype=np.uint64), 8)   # bit above num_qubits
    ham = rq.PauliSumXZ.from_xz(np.array([1], dtype=np.uint64), np.array([0], dtype=np.uint64),
                                np.array([1.0]), 8)
    space = rq.Subspace.from_u64(np.arange(4, dtype=np.uint64), 9)
    with pytest.raises(ValueError, match='qubits'):
        rq.SQDOperator(ham, space)
