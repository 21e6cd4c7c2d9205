"""GPU results at the full benchmark sizes checked against the CPU oracle's matvec.

* C2 (32 qubits, D = 262,144): every row of Hv from the cached product-layout kernels (FP64 and
  the complex64 bulk path) and from the on-the-fly diagonal kernel of the default cache
  strategy (1, 0), against the oracle's matvec on all rows; and the GPU eigenpair's residual
  ``||H v - E v|| / |E|`` with H applied by the oracle.
* C3 (48 qubits, D = 16,777,216) and C5 (40 qubits, D = 1,048,576): Hv on 2,048 seeded sample
  rows (all terms), and at C3 the mixed-precision eigenpair: its residual on those rows with H
  applied by the oracle, bounded by the reference's own convergence bound (the norm over any
  subset of rows is at most the full norm), and its energy against the FP64 path.

The oracle matvec here is ``oracle.cpu_baseline.CpuMatvecSample`` (the reference's
apply_h_x_cached + get_diagonal, sqd.py:603-709, with a sorted-search source lookup), itself
checked against the reference's own outputs in ``tests/test_oracle_cpu_baseline.py``.
Tolerances: FP64 paths 1e-13 of the largest |Hv| entry (summation order differs); complex64
elements and vectors 2e-6; eigenpair residual 1e-8 relative to |E|.
"""
import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import workloads as W
from oracle.cpu_baseline import CpuMatvecSample

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-13
FP32_RTOL = 2e-6
RESIDUAL_RTOL = 1e-8
SAMPLE_ROWS = 2048


def _operator(wl, cache=(1, 2), layout=None):
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, wl.num_qubits, force_real=True,
                                padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(wl.states, wl.num_qubits),
                        cache_strategy=cache)
    if layout is not None:
        for prec in (0, 1):
            op.set_layout(prec, layout)
    return op


def _oracle_rows(wl, rows, vectors):
    cpu = CpuMatvecSample(wl.x, wl.z, wl.coeffs, wl.states, rows)
    try:
        return [cpu.matvec(v) for v in vectors]
    finally:
        cpu.close()


def _err(got, ref):
    return np.abs(np.asarray(got) - ref).max() / np.abs(ref).max()


@pytest.fixture(scope='module')
def c2():
    return W.c2(0)


def test_c2_full_matvec_matches_oracle_on_every_row(c2):
    n = c2.states.shape[0]
    v = c2.start_vector(np.complex128)
    (ref,) = _oracle_rows(c2, np.arange(n), [v])
    vd = torch.as_tensor(v, device='cuda')
    op = _operator(c2, (1, 2), layout='product')
    hv64 = op.matvec(vd).cpu().numpy()
    assert _err(hv64, ref) < FP64_RTOL
    hv32 = op.matvec(vd.to(torch.complex64)).cpu().numpy()
    assert _err(hv32, ref) < FP32_RTOL
    op.set_layout(0, 'csr')
    assert _err(op.matvec(vd).cpu().numpy(), ref) < FP64_RTOL
    del op
    # the reference's default cache strategy: cached sources, diagonals computed per matvec
    op10 = _operator(c2, (1, 0))
    assert _err(op10.matvec(vd).cpu().numpy(), ref) < FP64_RTOL


@pytest.mark.parametrize('mode', ['fp64', 'mixed'])
def test_c2_eigenpair_residual_through_the_oracle_matvec(c2, mode):
    op = _operator(c2, (1, 2))
    op.autotune(torch.complex128)
    op.autotune(torch.complex64)
    x0 = torch.as_tensor(c2.start_vector(np.complex128), device='cuda')
    e, vec, _ = rq.ground_locg(op, x0, mode=mode)      # the reference's default tolerance
    v = vec.cpu().numpy()
    n = c2.states.shape[0]
    (hv,) = _oracle_rows(c2, np.arange(n), [v])
    res = np.linalg.norm(hv - e * v) / abs(e)
    assert res <= RESIDUAL_RTOL, res


def _sampled_rows_case(wl, layout, eigen=False):
    n = wl.states.shape[0]
    rows = np.sort(np.random.default_rng(1).choice(n, size=SAMPLE_ROWS, replace=False))
    v = wl.start_vector(np.complex128)
    op = _operator(wl, (1, 2), layout=layout)
    vd = torch.as_tensor(v, device='cuda')
    hv64 = op.matvec(vd).cpu().numpy()[rows]
    hv32 = op.matvec(vd.to(torch.complex64)).cpu().numpy()[rows]
    vectors = [v]
    sol = None
    if eigen:
        e, vec, _ = rq.ground_locg(op, vd, mode='mixed')
        e64, _, _ = rq.ground_locg(op, vd, mode='fp64')
        assert abs(e - e64) <= RESIDUAL_RTOL * abs(e64)
        # the reference's stopping test (ground_locg.py:371-376, tol = dtype epsilon):
        # |r| < eps * 10 * N * (|Hx| - theta)
        hx_norm = torch.linalg.vector_norm(op.matvec(vec)).item()
        bound = np.finfo(np.float64).eps * 10 * n * (hx_norm - e)
        sol = (e, vec.cpu().numpy(), bound)
        vectors.append(sol[1])
    del op, vd
    refs = _oracle_rows(wl, rows, vectors)
    assert _err(hv64, refs[0]) < FP64_RTOL
    assert _err(hv32, refs[0]) < FP32_RTOL
    if eigen:
        e, x, bound = sol
        # every subset of the residual's entries is bounded by its full norm
        res = np.linalg.norm(refs[1] - e * x[rows])
        assert res <= bound, (res, bound)


def test_c3_sampled_rows_and_mixed_eigenpair_match_oracle():
    _sampled_rows_case(W.c3(0), 'product', eigen=True)
    rq._lib.trim_memory()


def test_c5_sampled_rows_match_oracle():
    _sampled_rows_case(W.c5(0), None)
