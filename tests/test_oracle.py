"""Pins of the CPU oracle: against independent dense Kronecker-product matrices, numpy eigh,
the literal sort-based get_xsource, and the committed golden fixtures."""
import os

import numpy as np
import pytest

from rqutils_b200 import workloads as W
from oracle import symplectic as OS, sqd as OQ, dense as OD, ground_locg as OL

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def test_symplectic_matmul_matches_kronecker():
    rng = np.random.default_rng(1)
    for n in (3, 6, 8):
        x, z, c = W.random_pauli_sum(n, 25, rng)
        labels = W.labels_from_xz(x, z, n)
        ham = OS.from_paulisum((labels, list(c)))
        v = rng.standard_normal(2 ** n) + 1j * rng.standard_normal(2 ** n)
        ref = OD.hamiltonian_matrix(labels, c) @ v
        np.testing.assert_allclose(OS.matmul(ham, v), ref, rtol=0, atol=1e-12)


def test_from_paulisum_merges_and_groups():
    labels = ['XZ', 'ZX', 'XZ', 'II', 'YY', 'XI', 'XX']
    coeffs = [1.0, 2.0, 0.5, 0.0, -1.0, 3.0, 0.25]
    ham = OS.from_paulisum((labels, coeffs))
    # zero coefficient dropped, XZ merged (1.5); groups by X ascending: ZX (x=01), XZ/XI (x=10),
    # YY/XX (x=11)
    assert ham.x.shape[0] == 3
    dense = OD.hamiltonian_matrix(labels, coeffs)
    v = np.arange(4) + 1j
    np.testing.assert_allclose(OS.matmul(ham, v), dense @ v, atol=1e-13)


def test_sqd_oracle_matches_dense_eigh_notebook_recipe():
    # The reference's own test recipe (tests/sqd.ipynb), scaled down, seeded.
    labels, coeffs, states = W.notebook_case(3, nq=8, nsample=400, nterm=40)
    e, vec, basis = OQ.sqd((labels, list(coeffs)), states)
    uniq = np.unique(states, axis=0)
    assert (basis == uniq).all()
    h = OD.projected_matrix(labels, coeffs, OQ.states_to_u64(uniq))
    e0, v0 = OD.ground_energy(h)
    assert abs(e - e0) < 1e-8 * abs(e0)
    assert abs(abs(np.vdot(v0, vec)) - 1) < 1e-6


def test_get_xsource_sort_based_equals_dictionary_lookup():
    rng = np.random.default_rng(4)
    labels, coeffs, states = W.notebook_case(5, nq=9, nsample=300, nterm=30)
    ham = OS.from_paulisum((labels, list(coeffs)), force_real=True, add_padding=True)
    sp = OQ.uniquify_states(OQ.pack_states(states), 350)
    real = sp[:, 0] != 255
    nu = int(real.sum())
    for x in ham.x:
        a = OQ.get_xsource(x, sp)
        b = OQ.get_xsource_dict(x, sp)
        assert (a[real] == b[real]).all()
        # Fill-in slots: closed form used by the CUDA path.
        size = sp.shape[0]
        xzero = not np.any(x)
        for i in range(nu, size):
            expect = (i + 1) - size if i + 1 < size else (nu if xzero else -1)
            assert a[i] == expect
    del rng


def test_small_eigensolvers_match_eigh():
    rng = np.random.default_rng(7)
    for _ in range(50):
        for k in (2, 3):
            a = rng.standard_normal((k, k)) + 1j * rng.standard_normal((k, k))
            h = a + a.conj().T
            val, vec = (OL.eigenpair_2x2 if k == 2 else OL.eigenpair_3x3)(h)
            w, u = np.linalg.eigh(h)
            assert abs(val - w[0]) < 1e-10 * max(1, abs(w[0]))
            assert abs(abs(np.vdot(u[:, 0], vec)) - 1) < 1e-8


def test_ground_locg_oracle_matches_eigh_and_orth():
    rng = np.random.default_rng(2)
    a = rng.standard_normal((60, 60)) + 1j * rng.standard_normal((60, 60))
    h = a + a.conj().T
    w, u = np.linalg.eigh(h)
    e, v, it = OL.ground_locg(h, 0, tol=1e-12)
    assert abs(e - w[0]) < 1e-9 * abs(w[0])
    e1, v1, _ = OL.ground_locg(h, 5, orth=(u[:, 0],), tol=1e-12)
    assert abs(e1 - w[1]) < 1e-8 * abs(w[1])


def test_jw_construction_matches_dense_fermions():
    def dense_jw(h1, h2):
        norb = h1.shape[0]
        nq = 2 * norb
        eye, zz = np.eye(2), np.diag([1., -1.])
        sm = np.array([[0, 1], [0, 0]], dtype=float)

        def lower(p):
            m = np.ones((1, 1))
            for q in range(nq - 1, -1, -1):
                m = np.kron(m, sm if q == p else (zz if q < p else eye))
            return m
        A = [lower(p) for p in range(nq)]
        H = np.zeros((2 ** nq,) * 2)
        for i in range(norb):
            for j in range(norb):
                for s in range(2):
                    H += h1[i, j] * A[i + norb * s].T @ A[j + norb * s]
        for i, j, k, l in np.ndindex(*(norb,) * 4):
            for s in range(2):
                for t in range(2):
                    H += 0.5 * h2[i, j, k, l] * (A[i + norb * s].T @ A[k + norb * t].T
                                                 @ A[l + norb * t] @ A[j + norb * s])
        return H

    for norb in (2, 3):
        h1, h2 = W.random_integrals(norb, np.random.default_rng(norb))
        assert np.allclose(h2, h2.transpose(1, 0, 2, 3))
        assert np.allclose(h2, h2.transpose(2, 3, 0, 1))
        x, z, c = W.jw_hamiltonian(h1, h2)
        hp = OD.hamiltonian_matrix(W.labels_from_xz(x, z, 2 * norb), c)
        np.testing.assert_allclose(hp, dense_jw(h1, h2), atol=1e-12)


def test_label_mask_round_trip():
    rng = np.random.default_rng(3)
    x, z, _ = W.random_pauli_sum(20, 100, rng)
    labels = W.labels_from_xz(x, z, 20)
    x2, z2, n = W.xz_from_labels(labels)
    assert n == 20 and (x2 == x).all() and (z2 == z).all()


def test_state_packing_order_matches_reference_bytes():
    rng = np.random.default_rng(9)
    states = rng.integers(0, 2, size=(500, 13)).astype(np.uint8)
    packed = OQ.pack_states(states)
    vals = OQ.states_to_u64(states)
    # lexicographic order of padded big-endian rows == ascending uint64
    order_bytes = np.lexsort(tuple(packed[:, b] for b in range(packed.shape[1] - 1, -1, -1)))
    order_u64 = np.argsort(vals, kind='stable')
    assert (vals[order_bytes] == vals[order_u64]).all()
    assert (OQ.packed_to_u64(packed, 13) == vals).all()


@pytest.mark.parametrize('name', ['paulis_small', 'sqd_small', 'notebook_small'])
def test_oracle_reproduces_golden_fixtures(name):
    from tests.golden import make_golden as MG
    data = np.load(os.path.join(GOLDEN, name + '.npz'), allow_pickle=False)
    fresh = MG.CASES[name]()
    for key in data.files:
        a, b = data[key], fresh[key]
        if a.dtype.kind in 'fc':
            np.testing.assert_allclose(b, a, rtol=1e-12, atol=1e-12, err_msg=key)
        else:
            np.testing.assert_array_equal(b, a, err_msg=key)


def test_product_subspace_source_structure():
    """The invariant behind the product layout and the per-half connectivity, checked with the
    literal sort-based get_xsource (sqd.py:485-548): in an alpha x beta product subspace a
    group acting on one half has a source exactly when that half's string has a partner, and
    the source keeps the other half; a group acting on both halves needs both partners."""
    wl = W.jw_workload('t', 6, 2, 9, 11, 5)
    n, half = wl.num_qubits, wl.num_qubits // 2
    lo_mask = np.uint64((1 << half) - 1)
    states = np.sort(wl.states)
    sp = OQ.pack_states(OQ.u64_to_states(states, n))
    his = np.unique(states >> np.uint64(half))
    los = np.unique(states & lo_mask)
    nl = los.shape[0]
    assert his.shape[0] * nl == states.shape[0]
    oham = OS.from_paulisum((wl.labels, list(wl.coeffs)), force_real=True, add_padding=True)
    for xpacked in oham.x:
        src = OQ.get_xsource(xpacked, sp)[:states.shape[0]]
        x = int(OQ.packed_to_u64(xpacked[None, :], n)[0])
        xh, xl = x >> half, x & int(lo_mask)
        for r, s in enumerate(states):
            h, l = r // nl, r % nl
            ph = np.searchsorted(his, (int(s) >> half) ^ xh)
            pl = np.searchsorted(los, (int(s) & int(lo_mask)) ^ xl)
            ok_h = ph < his.shape[0] and his[ph] == ((int(s) >> half) ^ xh)
            ok_l = pl < nl and los[pl] == ((int(s) & int(lo_mask)) ^ xl)
            expect = ph * nl + pl if (ok_h and ok_l) else -1
            assert src[r] == expect


def _uniquify_indices_literal(states_p, states_size):
    """The index arithmetic of uniquify_states (sqd.py:457-481) transcribed step by step:
    stable lexsort, is_unique over positions 1..N-1, cumsum(bincount(cumsum)), -1 past the
    unique count."""
    keys = tuple(states_p[:, b] for b in range(states_p.shape[1] - 1, -1, -1))
    perm = np.lexsort(keys)
    srt = states_p[perm]
    is_unique = np.any(srt[1:] != srt[:-1], axis=1)
    total_unique = int(is_unique.sum()) + 1
    counts = np.bincount(np.cumsum(is_unique), minlength=states_size)[:states_size]
    idx_unique = np.cumsum(counts)
    idx_unique = np.where(np.arange(states_size) < total_unique, idx_unique, -1)
    return np.where(idx_unique >= 0, perm[np.clip(idx_unique, 0, None)], -1)


def test_uniquify_states_keeps_last_occurrence():
    rng = np.random.default_rng(12)
    bits = rng.integers(0, 2, size=(400, 7)).astype(np.uint8)     # many repeats of 128 strings
    sp = OQ.pack_states(bits)
    n_u = np.unique(sp, axis=0).shape[0]
    for size in (n_u, n_u + 9, n_u - 5, 400):
        rows, idx = OQ.uniquify_states(sp, size, return_indices=True)
        assert (idx == _uniquify_indices_literal(sp, size)).all()
        kept = idx >= 0
        assert (rows[kept] == sp[idx[kept]]).all()
        assert (rows[~kept] == 255).all()
        # last occurrence: no later input row repeats a kept row
        for i in np.flatnonzero(kept)[:40]:
            later = sp[idx[i] + 1:]
            assert not np.any(np.all(later == rows[i], axis=1))


def test_get_xsource_unsorted_input_restatement():
    rng = np.random.default_rng(13)
    bits = np.unique(rng.integers(0, 2, size=(300, 10)).astype(np.uint8), axis=0)
    sp = OQ.pack_states(bits)
    perm = rng.permutation(sp.shape[0])
    rows = sp[perm]
    for x in (OQ.pack_states(rng.integers(0, 2, size=(1, 10)).astype(np.uint8))[0]
              for _ in range(6)):
        got = OQ.get_xsource_unsorted(x, rows)
        table = {r.tobytes(): i for i, r in enumerate(rows)}
        expect = [table.get(np.bitwise_xor(r, x).tobytes(), -1) for r in rows]
        assert (got == np.array(expect)).all()
