"""The persistent LOCG launch (one kernel per loop: a thread-block cluster for small operators,
a cooperative grid otherwise) against the same fast iteration run as a CUDA graph of separate
passes (``SQD_LOCG_PERSISTENT=0``).

The persistent form fuses the second projection round, the matvec and the Gram dots into one
phase (A p is formed from A p0 and the carried A x, A y) and moves 16 bytes of every vector per
thread step, so the two forms round differently in the FP32 sweeps; after the FP64 polish their
energies must agree with each other and with the FP64 reference iteration to 1e-12 relative.
C1 (2,000 rows) runs as a cluster, C5 (1,048,576 rows of about one stored pair) as a
cooperative grid with one lane per row.
"""
import os

import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import workloads as W

pytestmark = pytest.mark.gpu

ENERGY_RTOL = 1e-12


def _solve(op, x0, mode, persistent):
    old = os.environ.get('SQD_LOCG_PERSISTENT')
    os.environ['SQD_LOCG_PERSISTENT'] = '1' if persistent else '0'
    try:
        return rq.ground_locg(op, x0, mode=mode)
    finally:
        if old is None:
            del os.environ['SQD_LOCG_PERSISTENT']
        else:
            os.environ['SQD_LOCG_PERSISTENT'] = old


@pytest.mark.parametrize('name', ['c1', 'c5'])
def test_persistent_iteration_matches_graph_form(name):
    wl = getattr(W, name)(0)
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, wl.num_qubits, force_real=True,
                                padded=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(wl.states, wl.num_qubits),
                        cache_strategy=(1, 2))
    x0 = torch.as_tensor(wl.start_vector(np.complex128), device='cuda')
    e64, _, _ = rq.ground_locg(op, x0, mode='fp64')
    ep, vp, itp = _solve(op, x0, 'mixed', True)
    rp = rq.ground_locg.last_residual
    eg, vg, itg = _solve(op, x0, 'mixed', False)
    rg = rq.ground_locg.last_residual
    assert abs(ep - eg) <= ENERGY_RTOL * abs(eg), (ep, eg)
    assert abs(ep - e64) <= ENERGY_RTOL * abs(e64), (ep, e64)
    # both stop on the reference's residual test
    assert rp <= 10 * rg + 1e-12 and rg <= 10 * rp + 1e-12, (rp, rg)
    assert abs(itp - itg) <= 0.25 * itg + 5, (itp, itg)
    assert abs(float(torch.linalg.vector_norm(vp)) - 1.0) < 1e-12
