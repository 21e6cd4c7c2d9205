"""Batched instances: the batched mixed-precision solver agrees per instance with the
single-instance FP64 solver (1e-8 relative), with the lowest eigenvalue of the oracle's sparse
projected matrix for every instance, and with dense eigh where the subspace is small."""
import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import workloads as W
from rqutils_b200.batched import SQDBatch, solve_instances
from oracle import dense as OD
from oracle.cpu_baseline import projected_csr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def instances():
    structure = W.JWStructure(16)
    dims = [(40, 30), (64, 48), (23, 90), (100, 70), (12, 15)]
    return [W.jw_workload(f'b{i}', 16, 4, a, b, 500 + i, structure)
            for i, (a, b) in enumerate(dims)]


def _op(inst):
    ham = rq.PauliSumXZ.from_xz(inst.x, inst.z, inst.coeffs, 32, force_real=True, padded=True)
    return rq.SQDOperator(ham, rq.Subspace.from_u64(inst.states, 32), cache_strategy=(1, 2))


def test_batched_solve_matches_single_instance_fp64(instances):
    ops = [_op(w) for w in instances]
    starts = [op.vinit() for op in ops]
    ref = [rq.ground_locg(op, s0)[0] for op, s0 in zip(ops, starts)]
    batch = SQDBatch(ops)
    assert batch.total_rows == sum(w.states.shape[0] for w in instances)
    for graph in (True, False):
        e, vecs, it, res = batch.solve(xinit_index=starts, use_graph=graph)
        for k in range(len(ops)):
            assert abs(e[k] - ref[k]) <= 1e-8 * abs(ref[k]), (k, e[k], ref[k])
            # the returned vector is a Ritz vector of that instance
            v = vecs[k].to(torch.complex128)
            rq_val = (torch.vdot(v, ops[k].matvec(v)) / torch.vdot(v, v)).real.item()
            assert abs(rq_val - e[k]) <= 1e-8 * abs(e[k])


def test_batched_smallest_instance_against_dense(instances):
    w = instances[-1]
    e, _ = solve_instances([w])
    h = OD.projected_matrix(W.labels_from_xz(w.x, w.z, 32), w.coeffs, w.states)
    e0 = np.linalg.eigvalsh(h)[0]
    assert abs(e[0] - e0) <= 1e-8 * abs(e0)


def test_wave_scheduler_splits_by_budget(instances):
    e_all, _ = solve_instances(instances)
    e_waves, _ = solve_instances(instances, budget_bytes=1 << 20)   # one instance per wave
    e_alone, _ = solve_instances(instances, alone_pairs=0)          # every instance alone
    np.testing.assert_allclose(e_waves, e_all, rtol=1e-8)
    np.testing.assert_allclose(e_alone, e_all, rtol=1e-8)


def test_batched_every_instance_against_the_oracle_matrix(instances):
    """Each instance's batched energy against the lowest eigenvalue of the oracle's projected
    sparse matrix (ARPACK, 1e-12 tolerance), 1e-8 relative."""
    from scipy.sparse.linalg import eigsh
    e, _ = solve_instances(instances)
    for k, w in enumerate(instances):
        h = projected_csr(w.x, w.z, w.coeffs, w.states)
        e0 = eigsh(h, k=1, which='SA', tol=1e-12)[0][0]
        assert abs(e[k] - e0) <= 1e-8 * abs(e0), (k, e[k], e0)
