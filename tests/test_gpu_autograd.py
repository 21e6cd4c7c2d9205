"""Gradients through the SQD operator: the hand-written backward of the matvec (checked with
torch.autograd.gradcheck) and the Hellmann-Feynman ground-energy gradient (checked against
central finite differences and the NumPy restatement)."""
import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import workloads as W
from rqutils_b200.autograd import hamiltonian_matvec, ground_energy
from oracle import dense as OD

pytestmark = pytest.mark.gpu


def _small_case(seed=0, n=10, m=40, d=120, k=5):
    rng = np.random.default_rng(seed)
    x, z, c = W.random_pauli_sum(n, m, rng, scale=0.5)
    states = W.weight_subspace(n, k, d, rng)
    ham = rq.PauliSumXZ.from_xz(x, z, c, n, force_real=True, padded=True)
    space = rq.Subspace.from_u64(states, n)
    return x, z, c, states, ham, space


def test_set_coeffs_matches_fresh_operator():
    x, z, c, states, ham, space = _small_case(1)
    op = rq.SQDOperator(ham, space, cache_strategy=(1, 2))
    c2 = c * 1.7 - 0.1 * np.sign(c)
    ham.set_coeffs(torch.as_tensor(c2))
    op.refresh()
    fresh = rq.SQDOperator(rq.PauliSumXZ.from_xz(x, z, c2, 10, force_real=True), space,
                           cache_strategy=(1, 2))
    v = torch.randn(space.states_size, dtype=torch.complex128, device='cuda')
    torch.testing.assert_close(op.matvec(v), fresh.matvec(v), rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize('cache', [(1, 0), (1, 2)])
def test_matvec_backward_gradcheck(cache):
    x, z, c, states, ham, space = _small_case(2, m=25, d=60)
    op = rq.SQDOperator(ham, space, cache_strategy=cache)
    coeffs = torch.as_tensor(c, device='cuda').clone().requires_grad_(True)
    v = torch.randn(space.states_size, dtype=torch.complex128, device='cuda',
                    requires_grad=True)
    assert torch.autograd.gradcheck(lambda cc, vv: hamiltonian_matvec(cc, vv, op),
                                    (coeffs, v), eps=1e-6, atol=1e-7, rtol=1e-6)


def test_ground_energy_gradient_matches_finite_differences_and_hellmann_feynman():
    x, z, c, states, ham, space = _small_case(3, n=12, m=60, d=400, k=6)
    op = rq.SQDOperator(ham, space, cache_strategy=(1, 2))
    coeffs = torch.as_tensor(c, device='cuda').clone().requires_grad_(True)
    e = ground_energy(coeffs, op)
    e.backward()
    grad = coeffs.grad.cpu().numpy()
    # dense oracle: eigenvector of the projected matrix, <v|P_r|v> per raw term
    labels = W.labels_from_xz(x, z, 12)
    h = OD.projected_matrix(labels, c, states)
    w, u = np.linalg.eigh(h)
    assert abs(e.item() - w[0]) < 1e-9 * abs(w[0])
    hf = np.array([np.real(np.vdot(u[:, 0], OD.projected_matrix([lab], [1.0], states)
                                   @ u[:, 0])) for lab in labels])
    np.testing.assert_allclose(grad, hf, rtol=1e-6, atol=1e-8)
    # central differences on a few coordinates (h = 1e-5), FP64 LOCG at the default tolerance
    rng = np.random.default_rng(0)
    hstep = 1e-5
    for k in rng.choice(len(c), size=6, replace=False):
        cp, cm = c.copy(), c.copy()
        cp[k] += hstep
        cm[k] -= hstep
        ep = ground_energy(torch.as_tensor(cp, device='cuda'), op).item()
        em = ground_energy(torch.as_tensor(cm, device='cuda'), op).item()
        fd = (ep - em) / (2 * hstep)
        assert abs(fd - grad[k]) <= 1e-6 * max(1.0, abs(grad[k])) + 1e-7, (k, fd, grad[k])
