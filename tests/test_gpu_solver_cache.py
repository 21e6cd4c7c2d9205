"""Solver objects cached on an operator between LOCG solves: repeated solves, solves after a
change of the matvec schedule or of the coefficients, and solves on another stream must give
the results of a fresh operator."""
import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _case(seed=2):
    wl = W.jw_workload('jw_small', 8, 3, 20, 24, seed)
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, wl.num_qubits, force_real=True,
                                padded=True)
    space = rq.Subspace.from_u64(wl.states, wl.num_qubits)
    return wl, ham, space


@pytest.mark.parametrize('mode', ['fp64', 'mixed'])
def test_repeated_solves_reuse_and_stay_exact(mode):
    wl, ham, space = _case()
    op = rq.SQDOperator(ham, space, cache_strategy=(1, 2))
    x0 = torch.as_tensor(wl.start_vector(), device='cuda')
    e1, v1, it1 = rq.ground_locg(op, x0, mode=mode)
    e2, v2, it2 = rq.ground_locg(op, x0, mode=mode)
    assert e1 == e2 and it1 == it2                      # deterministic reductions, same path
    torch.testing.assert_close(v1, v2, rtol=0, atol=0)
    # schedule changes between solves: the cached graphs are rebuilt
    op.set_lanes(0, 4)
    op.set_lanes(1, 8)
    op.set_layout(0, 'product')
    op.set_layout(1, 'product')
    e3, _, _ = rq.ground_locg(op, x0, mode=mode)
    assert abs(e3 - e1) <= 1e-12 * abs(e1)
    # another stream
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        e4, _, _ = rq.ground_locg(op, x0, mode=mode)
    torch.cuda.synchronize()
    assert abs(e4 - e1) <= 1e-12 * abs(e1)


def test_cached_solver_follows_coefficient_refresh():
    wl, ham, space = _case(5)
    op = rq.SQDOperator(ham, space, cache_strategy=(1, 2))
    x0 = torch.as_tensor(wl.start_vector(), device='cuda')
    rq.ground_locg(op, x0, mode='mixed')
    c2 = wl.coeffs * 0.8 + 0.01 * np.sign(wl.coeffs)
    ham.set_coeffs(torch.as_tensor(c2))
    op.refresh()
    e_cached, _, _ = rq.ground_locg(op, x0, mode='mixed')
    fresh = rq.SQDOperator(rq.PauliSumXZ.from_xz(wl.x, wl.z, c2, wl.num_qubits, force_real=True,
                                                 padded=True), space, cache_strategy=(1, 2))
    e_fresh, _, _ = rq.ground_locg(fresh, x0, mode='mixed')
    assert abs(e_cached - e_fresh) <= 1e-12 * abs(e_fresh)


def test_mixed_precision_excited_state_with_orth():
    """Deflation against the ground state (ground_locg's orth) in the mixed-precision solver:
    FP32 sweeps project every search direction, the FP64 polish runs the reference iteration."""
    wl, ham, space = _case(7)
    op = rq.SQDOperator(ham, space, cache_strategy=(1, 2))
    ip, ix, dt = op.csr()
    n = op.size
    dense = np.zeros((n, n), dtype=np.complex128)
    ipn, ixn, dtn = ip.cpu().numpy(), ix.cpu().numpy(), dt.cpu().numpy()
    for r in range(n):
        dense[r, ixn[ipn[r]:ipn[r + 1]]] += dtn[ipn[r]:ipn[r + 1]]
    w, u = np.linalg.eigh(dense)
    assert w[1] - w[0] > 1e-6
    x0 = torch.as_tensor(wl.start_vector(), device='cuda')
    orth = (torch.as_tensor(u[:, 0], device='cuda'),)
    e64, v64, _ = rq.ground_locg(op, x0, orth=orth, mode='fp64', tol=1e-12)
    e32, v32, _ = rq.ground_locg(op, x0, orth=orth, mode='mixed', tol=1e-12)
    assert abs(e64 - w[1]) <= 1e-8 * abs(w[1])
    assert abs(e32 - w[1]) <= 1e-8 * abs(w[1])
    assert abs(np.vdot(u[:, 0], v32.cpu().numpy())) < 1e-6
    # the cached solver objects of an unconstrained solve are unaffected
    e_gs, _, _ = rq.ground_locg(op, x0, mode='mixed')
    assert abs(e_gs - w[0]) <= 1e-8 * abs(w[0])


def test_promoted_element_cache_gives_the_same_results():
    """SQDOptions.promote_cache: an operator built with the reference's default (1, 0) caches
    its elements ((1, 2), product layout on a product subspace); Hv and the sqd energy agree
    with the on-the-fly diagonals."""
    wl = W.c2_small(0, 96, 80)
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, 32, force_real=True, padded=True)
    space = rq.Subspace.from_u64(wl.states, 32)
    op = rq.SQDOperator(ham, space, cache_strategy=(1, 0))
    v = torch.as_tensor(wl.start_vector(np.complex128), device='cuda')
    hv10 = op.matvec(v).cpu().numpy()
    assert op.promote_cache() and op.cache_strategy == (1, 2)
    assert op.get_layout(0) == 'product' and op.get_layout(1) == 'product'
    hv12 = op.matvec(v).cpu().numpy()
    assert np.abs(hv12 - hv10).max() <= 1e-13 * np.abs(hv10).max()
    shifts = np.arange(31, -1, -1, dtype=np.uint64)
    bits = ((wl.states[:, None] >> shifts[None, :]) & np.uint64(1)).astype(np.uint8)
    e_on = rq.sqd((wl.labels, list(wl.coeffs)), bits, options={'promote_cache': False,
                                                                'return_eigvec': False})
    e_pr = rq.sqd((wl.labels, list(wl.coeffs)), bits, options={'return_eigvec': False})
    assert abs(e_on - e_pr) <= 1e-12 * abs(e_on)
