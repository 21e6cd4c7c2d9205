"""Product-subspace layout of the cached matvec (dense high-half / low-half slabs plus CSR
lists for the two-half pairs) against the CSR layout and the CPU oracle (apply_h_x_cached,
sqd.py:694-709)."""
import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import workloads as W
from rqutils_b200._lib import SQDError
from oracle import symplectic as OS, sqd as OQ

pytestmark = pytest.mark.gpu

# FP64 layouts sum a row in different orders: agreement to a few ulps of the row sums.
MATVEC_RTOL = 1e-13
MATVEC32_RTOL = 2e-6
PREC = {torch.complex128: 0, torch.float64: 0, torch.complex64: 1, torch.float32: 1}


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _jw_small(seed=0):
    """JW Hamiltonian of 8 orbitals (16 qubits) on a 24 x 20 product of 3-electron strings."""
    return W.jw_workload('jw_small', 8, 3, 20, 24, seed)


def _oracle_hv(x, z, c, states, n, v, force_real):
    labels = W.labels_from_xz(x, z, n)
    oham = OS.from_paulisum((labels, list(c)), force_real=force_real, add_padding=True)
    sp = OQ.pack_states(OQ.u64_to_states(states, n))
    xs = np.stack([OQ.get_xsource(xm, sp) for xm in oham.x])
    return OQ.apply_h_x_cached(v.astype(np.complex128), xs, oham.z, oham.c, sp)


def _vector(size, dtype, seed=3):
    g = torch.Generator().manual_seed(seed)
    v = torch.randn(size, generator=g, dtype=torch.float64)
    if dtype.is_complex:
        v = v + 1j * torch.randn(size, generator=g, dtype=torch.float64)
    return v.to(dtype).cuda()


@pytest.mark.parametrize('dtype', [torch.complex128, torch.complex64, torch.float64,
                                   torch.float32])
def test_product_layout_matches_csr_and_oracle(dtype):
    wl = _jw_small()
    n = wl.num_qubits
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, n, force_real=True, padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(wl.states, n), cache_strategy=(1, 2))
    info = op.product_info()
    assert (info['n_high'], info['n_low']) == (24, 20)
    assert info['pairs_high'] == -1
    v = _vector(op.size, dtype)
    prec = PREC[dtype]
    csr = op.matvec(v).cpu().numpy()
    ref = _oracle_hv(wl.x, wl.z, wl.coeffs, wl.states, n, v.cpu().numpy(), True)
    tol = MATVEC_RTOL if prec == 0 else MATVEC32_RTOL
    for layout in ('product', 'product-csr'):
        op.set_layout(prec, layout)
        assert op.get_layout(prec) == layout and op.get_layout(1 - prec) == 'csr'
        info = op.product_info()
        assert info['pairs_high'] + info['pairs_low'] + info['pairs_mixed'] == op.nnz
        assert min(info['pairs_high'], info['pairs_low'], info['pairs_mixed']) > 0
        for lanes in (1, 4, 32):
            for chunk in (0, 64):
                op.set_lanes(prec, lanes)
                op.set_chunk(prec, chunk)
                got = op.matvec(v).cpu().numpy()
                assert rel(got, ref) < tol
                assert rel(got, csr) < (MATVEC_RTOL if prec == 0 else MATVEC32_RTOL)


@pytest.mark.parametrize('dtype', [torch.complex128, torch.complex64])
def test_product_layout_complex_elements(dtype):
    rng = np.random.default_rng(11)
    x, z, c = W.random_pauli_sum(16, 500, rng, wmax=4)
    states = W.product_subspace(8, 4, 30, 22, rng)
    ham = rq.PauliSumXZ.from_xz(x, z, c, 16, padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(states, 16), cache_strategy=(1, 2))
    assert op.value_complex
    v = _vector(op.size, dtype, seed=5)
    ref = _oracle_hv(x, z, c, states, 16, v.cpu().numpy(), False)
    for layout in ('product', 'product-csr'):
        op.set_layout(PREC[dtype], layout)
        got = op.matvec(v).cpu().numpy()
        assert rel(got, ref) < (MATVEC_RTOL if PREC[dtype] == 0 else MATVEC32_RTOL)


def test_product_layout_without_two_half_pairs_or_diagonal():
    """Terms on one half only (no two-half pairs) and no Z-only group (no diagonal entry)."""
    rng = np.random.default_rng(4)
    xl, zl, cl = W.random_pauli_sum(8, 60, rng, wmin=1, wmax=3)
    xh, zh, ch = W.random_pauli_sum(8, 60, rng, wmin=1, wmax=3)
    keep_l, keep_h = xl != 0, xh != 0
    x = np.concatenate([xl[keep_l], xh[keep_h] << np.uint64(8)])
    z = np.concatenate([zl[keep_l], zh[keep_h] << np.uint64(8)])
    c = np.concatenate([cl[keep_l], ch[keep_h]])
    states = W.product_subspace(8, 4, 25, 33, rng)
    ham = rq.PauliSumXZ.from_xz(x, z, c, 16, force_real=True, padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(states, 16), cache_strategy=(1, 2))
    v = _vector(op.size, torch.complex128, seed=9)
    ref = _oracle_hv(x, z, c, states, 16, v.cpu().numpy(), True)
    for prec, dt in ((0, torch.complex128), (1, torch.complex64)):
        op.set_layout(prec, 'product')
        got = op.matvec(v.to(dt)).cpu().numpy()
        assert rel(got, ref) < (MATVEC_RTOL if prec == 0 else MATVEC32_RTOL)
    assert op.product_info()['pairs_mixed'] == 0


def test_product_layout_rejected_for_other_subspaces():
    wl = W.c1(0)                                   # weight-8 strings: not a product
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, 16, force_real=True, padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(wl.states, 16), cache_strategy=(1, 2))
    assert op.product_info()['n_high'] == 0 and not op.has_product_layout
    with pytest.raises(SQDError):
        op.set_layout(0, 'product')
    assert op.get_layout(0) == 'csr'
    # a product subspace with fill-in slots is refused too
    jw = _jw_small()
    hj = rq.PauliSumXZ.from_xz(jw.x, jw.z, jw.coeffs, 16, force_real=True, padded=True)
    sp = rq.Subspace.from_u64(jw.states, 16, states_size=jw.states.shape[0] + 7)
    opf = rq.SQDOperator(hj, sp, cache_strategy=(1, 2))
    with pytest.raises(SQDError):
        opf.set_layout(0, 'product')
    # uncached elements: no product layout
    opx = rq.SQDOperator(hj, rq.Subspace.from_u64(jw.states, 16), cache_strategy=(1, 0))
    assert not opx.has_product_layout


def test_product_layout_locg_autotune_and_refresh():
    wl = _jw_small(1)
    n = wl.num_qubits
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, n, force_real=True, padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(wl.states, n), cache_strategy=(1, 2))
    x0 = torch.as_tensor(wl.start_vector(), device='cuda')
    e_csr, _, _ = rq.ground_locg(op, x0, mode='fp64')
    tuned = op.autotune(layouts=('product',))
    assert tuned['fp64']['layout'] == 'product' and tuned['fp32']['layout'] == 'product'
    for mode in ('fp64', 'mixed'):
        e, _, _ = rq.ground_locg(op, x0, mode=mode)
        assert abs(e - e_csr) <= 1e-10 * abs(e_csr)
    # coefficient update: the slabs and the tail copies follow the refreshed elements
    c2 = wl.coeffs * 1.3
    ham.set_coeffs(torch.as_tensor(c2))
    op.refresh()
    v = _vector(op.size, torch.complex128, seed=2)
    ref = _oracle_hv(wl.x, wl.z, c2, wl.states, n, v.cpu().numpy(), True)
    for layout in ('product', 'product-csr'):
        op.set_layout(0, layout)
        op.set_layout(1, layout)
        assert rel(op.matvec(v).cpu().numpy(), ref) < MATVEC_RTOL
        assert rel(op.matvec(v.to(torch.complex64)).cpu().numpy(), ref) < MATVEC32_RTOL


def _connectivity_cases():
    wl = _jw_small(3)
    yield wl.x, wl.z, wl.coeffs, wl.states, True
    rng = np.random.default_rng(21)
    x, z, c = W.random_pauli_sum(16, 400, rng, wmax=4)
    yield x, z, c, W.product_subspace(8, 4, 27, 31, rng), False
    xl, zl, cl = W.random_pauli_sum(8, 50, rng, wmin=1, wmax=3)
    keep = xl != 0                                   # no Z-only terms: no diagonal group
    yield (np.concatenate([xl[keep], xl[keep] << np.uint64(8)]),
           np.concatenate([zl[keep], zl[keep] << np.uint64(8)]),
           np.concatenate([cl[keep], cl[keep]]), W.product_subspace(8, 4, 19, 23, rng), True)


@pytest.mark.parametrize('case', range(3))
def test_product_connectivity_equals_sweep(case):
    """Pairs assembled from per-half partner lists: the same CSR (row pointers, sources,
    elements, order) as the (row, group) sweep, bit for bit."""
    x, z, c, states, real = list(_connectivity_cases())[case]
    ham = rq.PauliSumXZ.from_xz(x, z, c, 16, force_real=real, padded=True)
    space = rq.Subspace.from_u64(states, 16)
    sweep = rq.SQDOperator(ham, space, cache_strategy=(1, 2), lookup='hash')
    prod = rq.SQDOperator(ham, space, cache_strategy=(1, 2), lookup='product')
    auto = rq.SQDOperator(ham, space, cache_strategy=(1, 2), lookup='auto')
    assert sweep.nnz == prod.nnz == auto.nnz
    a, b = sweep.csr(), prod.csr()
    for u, w in zip(a, b):
        np.testing.assert_array_equal(u.cpu().numpy(), w.cpu().numpy())
    v = _vector(sweep.size, torch.complex128, seed=case)
    torch.testing.assert_close(prod.matvec(v), sweep.matvec(v), rtol=0, atol=0)


def test_product_lookup_needs_a_product_subspace():
    wl = W.c1(0)
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, 16, force_real=True, padded=True)
    space = rq.Subspace.from_u64(wl.states, 16)
    with pytest.raises(SQDError):
        rq.SQDOperator(ham, space, cache_strategy=(1, 2), lookup='product')
    auto = rq.SQDOperator(ham, space, cache_strategy=(1, 2), lookup='auto')   # sweep fallback
    ref = rq.SQDOperator(ham, space, cache_strategy=(1, 2), lookup='hash')
    v = _vector(ref.size, torch.complex128)
    torch.testing.assert_close(auto.matvec(v), ref.matvec(v), rtol=0, atol=0)


def test_product_without_conserved_weights():
    """Halves of random strings (no conserved weight, so no sector filter): the per-half
    connectivity still equals the sweep's and the product layout still matches the oracle."""
    rng = np.random.default_rng(33)
    hi = np.unique(rng.integers(0, 256, size=40, dtype=np.uint64))
    lo = np.unique(rng.integers(0, 256, size=30, dtype=np.uint64))
    states = ((hi[:, None] << np.uint64(8)) | lo[None, :]).reshape(-1)
    x, z, c = W.random_pauli_sum(16, 300, rng, wmax=3)
    ham = rq.PauliSumXZ.from_xz(x, z, c, 16, force_real=True, padded=True)
    space = rq.Subspace.from_u64(states, 16)
    sweep = rq.SQDOperator(ham, space, cache_strategy=(1, 2), lookup='hash')
    prod = rq.SQDOperator(ham, space, cache_strategy=(1, 2), lookup='product')
    for u, w in zip(sweep.csr(), prod.csr()):
        np.testing.assert_array_equal(u.cpu().numpy(), w.cpu().numpy())
    v = _vector(prod.size, torch.complex128, seed=4)
    ref = _oracle_hv(x, z, c, states, 16, v.cpu().numpy(), True)
    for layout in ('product', 'product-csr'):
        prod.set_layout(0, layout)
        assert rel(prod.matvec(v).cpu().numpy(), ref) < MATVEC_RTOL


def test_product_layout_large_grid_matches_csr():
    """1024 x 512 product (multi-panel slab passes with many slabs per panel): product layout
    against the CSR layout, both precisions."""
    rng = np.random.default_rng(8)
    hi = np.arange(1024, dtype=np.uint64)
    lo = np.sort(rng.choice(np.arange(1024, dtype=np.uint64), size=512, replace=False))
    states = ((hi[:, None] << np.uint64(10)) | lo[None, :]).reshape(-1)
    x, z, c = W.random_pauli_sum(20, 200, rng, wmax=3)
    ham = rq.PauliSumXZ.from_xz(x, z, c, 20, force_real=True, padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(states, 20), cache_strategy=(1, 2))
    info = op.product_info()
    assert (info['n_high'], info['n_low']) == (1024, 512)
    for dt, prec, tol in ((torch.complex128, 0, MATVEC_RTOL), (torch.complex64, 1, MATVEC32_RTOL)):
        v = _vector(op.size, dt, seed=6)
        op.set_layout(prec, 'csr')
        ref = op.matvec(v).to(torch.complex128).cpu().numpy()
        op.set_layout(prec, 'product-csr')
        got = op.matvec(v).to(torch.complex128).cpu().numpy()
        assert rel(got, ref) < tol


@pytest.mark.parametrize('seed, short', [(0, True), (2, False)])
def test_product_csr_tail_forms(seed, short):
    """Two-half pairs on the CSR tail kernel: a contiguous copy of the row tails when they are
    short (at most 32 pairs per row on average; seed 0: 31.8), the tails read in place inside the
    rows' pair lists otherwise (seed 2: 39.0).  Both against the oracle, every schedule, and after
    a coefficient refresh."""
    wl = _jw_small(seed)
    n = wl.num_qubits
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, n, force_real=True, padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(wl.states, n), cache_strategy=(1, 2))
    for prec in (0, 1):
        op.set_layout(prec, 'product-csr')
    assert (op.product_info()['pairs_mixed'] <= 32 * op.size) == short
    for coeffs in (wl.coeffs, wl.coeffs * 0.7 - 0.01):
        if coeffs is not wl.coeffs:
            ham.set_coeffs(torch.as_tensor(coeffs))
            op.refresh()
        v = _vector(op.size, torch.complex128, seed=seed + 1)
        ref = _oracle_hv(wl.x, wl.z, coeffs, wl.states, n, v.cpu().numpy(), True)
        for prec, dt, tol in ((0, torch.complex128, MATVEC_RTOL),
                              (1, torch.complex64, MATVEC32_RTOL)):
            for lanes in (1, 4, 32):
                for chunk in (0, 64):
                    op.set_lanes(prec, lanes)
                    op.set_chunk(prec, chunk)
                    assert rel(op.matvec(v.to(dt)).cpu().numpy(), ref) < tol


@pytest.mark.parametrize('dtype', [torch.complex64, torch.float32])
def test_fp32_slabs_with_unaligned_vectors(dtype):
    """FP32 slabs of even-sized halves read two positions per lane with paired vector loads;
    v and Hv that start off that alignment (views one element into a buffer) take the
    element-wise path, with the same sums bit for bit."""
    wl = _jw_small()
    n = wl.num_qubits
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, n, force_real=True, padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(wl.states, n), cache_strategy=(1, 2))
    op.set_layout(1, 'product')
    v = _vector(op.size, dtype, seed=8)
    ref = _oracle_hv(wl.x, wl.z, wl.coeffs, wl.states, n, v.cpu().numpy(), True)
    aligned = op.matvec(v)
    assert rel(aligned.cpu().numpy(), ref) < MATVEC32_RTOL
    vbuf = torch.zeros(op.size + 1, dtype=dtype, device='cuda')
    vbuf[1:] = v
    obuf = torch.zeros(op.size + 1, dtype=dtype, device='cuda')
    op.matvec(vbuf[1:], obuf[1:])
    assert torch.equal(obuf[1:], aligned)
    out = torch.zeros_like(v)
    op.matvec(vbuf[1:], out)                       # only the input off the pairing
    assert torch.equal(out, aligned)
