r"""Differentiation of the SQD operator and of its ground energy w.r.t. the Pauli coefficients.

Two ``torch.autograd.Function`` s with hand-written backwards:

* :func:`hamiltonian_matvec` — ``y = H(c) v``.  The adjoint w.r.t. ``v`` is ``H^dagger g`` (H is
  Hermitian, so the same CUDA matvec); the adjoint w.r.t. the raw coefficient ``c_r`` is the
  per-term reduction ``Re <g| P_t |v>`` (``sqd_grad_terms``) of the merged term ``t`` that
  ``c_r`` was summed into (PyTorch's conjugate-Wirtinger convention for a real parameter).
* :func:`ground_energy` — ``E0(c)`` from ``ground_locg``; by Hellmann-Feynman
  ``dE0/dc_r = <v0| P_t |v0>`` at the converged, normalised ground vector ``v0``.

The reference has no gradient path (its solver is a ``jax.lax.while_loop``); the only
differentiable object there is the matvec w.r.t. ``PauliSumXZ.c``, which is what these restate.
Raw terms whose coefficient was zero when the Pauli sum was created have no slot in the table
and get zero gradient.  Coefficients are the real raw coefficients (``force_real`` sums).
"""
import torch

from .ground_locg import ground_locg


def _apply_coeffs(op, coeffs):
    """Load ``coeffs`` into the operator's Pauli sum if they differ from the current ones."""
    current = getattr(op, '_coeffs', None)
    c = coeffs.detach().to(torch.float64)
    if current is None or current.shape != c.shape or not torch.equal(current, c.to(current.device)):
        op.hamiltonian.set_coeffs(c)
        op.refresh()
        op._coeffs = c.to(op.space.device).clone()


def _scatter_terms(op, g_terms):
    r2t = op.hamiltonian.raw_to_term()
    out = torch.zeros(r2t.shape[0], dtype=torch.float64, device=g_terms.device)
    ok = r2t >= 0
    out[ok] = g_terms[r2t[ok]]
    return out


class _Matvec(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coeffs, v, op):
        _apply_coeffs(op, coeffs)
        ctx.op = op
        ctx.save_for_backward(v)
        return op.matvec(v.contiguous())

    @staticmethod
    def backward(ctx, g):
        (v,) = ctx.saved_tensors
        op = ctx.op
        g = g.contiguous()
        gv = op.matvec(g.to(v.dtype)) if ctx.needs_input_grad[1] else None
        gc = None
        if ctx.needs_input_grad[0]:
            gc = _scatter_terms(op, op.grad_terms(g, v))
        return gc, gv, None


class _GroundEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coeffs, op, xinit, kwargs):
        _apply_coeffs(op, coeffs)
        e, vec, _ = ground_locg(op, xinit, **kwargs)
        vec = vec / torch.linalg.vector_norm(vec)
        ctx.op = op
        ctx.save_for_backward(vec)
        return torch.tensor(e, dtype=torch.float64, device=vec.device)

    @staticmethod
    def backward(ctx, g):
        (vec,) = ctx.saved_tensors
        op = ctx.op
        gc = _scatter_terms(op, op.grad_terms(vec, vec)) * g
        return gc, None, None, None


def hamiltonian_matvec(coeffs, v, op):
    """``H(coeffs) @ v`` for an :class:`~rqutils_b200.sqd.SQDOperator`, differentiable in both
    ``coeffs`` (raw real coefficients, one per term the Pauli sum was created from) and ``v``."""
    return _Matvec.apply(coeffs, v, op)


def ground_energy(coeffs, op, xinit=None, **locg_kwargs):
    """Ground energy ``E0(coeffs)`` (0-dim FP64 tensor) with the Hellmann-Feynman gradient.
    ``xinit`` defaults to the operator's ``vinit``; ``locg_kwargs`` go to ``ground_locg``."""
    if xinit is None:
        _apply_coeffs(op, coeffs)
        xinit = op.vinit()
    return _GroundEnergy.apply(coeffs, op, xinit, locg_kwargs)
