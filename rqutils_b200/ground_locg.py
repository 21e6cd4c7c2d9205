r"""Single-vector LOBPCG on a B200 (drop-in for ``rqutils.ground_locg``).

``ground_locg(mat, xinit, args=(), orth=(), maxiter=1000, tol=None, vspace=None, log_level)``
has the reference's signature and meaning (ground_locg.py:128-162) and returns
``(eigval, eigvec, niter)`` with ``eigvec`` a CUDA tensor.  ``mat`` may be

* an :class:`~rqutils_b200.sqd.SQDOperator`: the fused device solver (``csrc/locg.cu``), the
  whole while-loop captured as one CUDA graph;
* a callable ``mat(x, *args) -> Ax`` on CUDA tensors: the same device solver, calling back into
  Python for every matvec;
* a dense matrix (CUDA tensor or array): as the reference's ``_ground_locg_matrix``.

Two B200 extensions: ``mode='mixed'`` (FP32 sweeps + FP64 refinement, SQD operators only) and
``use_graph``.

``log_level <= logging.DEBUG`` prints the reference's per-iteration lines (ground_locg.py:330-331,
377-378: ``LOCG iteration {i}`` and ``Residual {r}, reltol {reltol}, converged: {c}``) after the
solve, from a record the device solver writes as it iterates (the loop itself runs on the GPU;
FP32 sweeps of the mixed solver print as ``FP32 sweep {i}`` lines first).  The rows are kept in
``ground_locg.last_history``: an array of (phase, iteration, theta, |r|, reltol, converged), phase
0 for FP64 iterations and 1 for FP32 sweeps.
"""
import logging

import numpy as np
import torch

from . import _lib


def ground_locg(mat, xinit, args=(), orth=(), maxiter=1000, tol=None, vspace=None,
                log_level=logging.WARNING, mode='fp64', use_graph=True):
    """Lowest eigenpair of a Hermitian operator (ground_locg.py:128-423)."""
    from .sqd import SQDOperator
    _lib.require_cuda()
    if not isinstance(orth, tuple):
        orth = (orth,)
    dev = torch.device('cuda', torch.cuda.current_device())
    dense = None
    if isinstance(mat, SQDOperator):
        n = mat.size
        if not isinstance(xinit, (int, np.integer)):
            dtype = torch.promote_types(torch.as_tensor(xinit).dtype, mat.dtype)
        elif vspace is not None:
            dtype = torch.promote_types(_torch_dtype(vspace[1]), mat.dtype)
        else:
            dtype = mat.dtype
    elif callable(mat):
        if isinstance(xinit, (int, np.integer)):
            if vspace is None:
                raise ValueError('vspace is required when mat is callable and xinit an int')
            n, dtype = int(vspace[0]), _torch_dtype(vspace[1])
        else:
            xt = torch.as_tensor(xinit)
            n, dtype = xt.shape[0], xt.dtype
    else:
        dense = torch.as_tensor(mat, device=dev)
        n = dense.shape[1]
        dtype = dense.dtype if isinstance(xinit, (int, np.integer)) else \
            torch.as_tensor(xinit).dtype
    if dtype not in (torch.float64, torch.complex128):
        dtype = torch.complex128 if dtype.is_complex else torch.float64
    if dense is not None:
        dense = dense.to(dtype)
        mat = None
    code = _lib.dtype_code(dtype)

    if isinstance(xinit, (int, np.integer)):
        xinit_t = None
        xinit_index = int(xinit)
        if xinit_index < 0 or xinit_index >= n:
            raise ValueError('xinit index out of range')
    else:
        xinit_t = torch.as_tensor(xinit, device=dev).to(dtype).contiguous()
        xinit_index = 0
        if xinit_t.shape[0] != n:
            raise ValueError('xinit length does not match the operator')

    orth_t = [torch.as_tensor(o, device=dev).to(dtype).contiguous() for o in orth]
    orth_arr = (_lib._vp * max(1, len(orth_t)))(*[o.data_ptr() for o in orth_t])

    keep = []
    if isinstance(mat, SQDOperator):
        fn = _lib._c.cast(_lib.load().sqd_op_matvec_cb, _lib._vp)
        ctx = mat.handle
        mode_code = _lib.SQD_LOCG_MIXED if mode == 'mixed' else _lib.SQD_LOCG_FP64
    else:
        if mode == 'mixed':
            raise ValueError("mode='mixed' needs an SQDOperator")
        mode_code = _lib.SQD_LOCG_FP64
        apply = (lambda x: dense @ x) if dense is not None else (lambda x: mat(x, *args))
        errors = []

        def _cb(_ctx, xp, yp, _stream):
            try:
                x = _lib.tensor_from_ptr(xp, n, dtype, dev)
                y = _lib.tensor_from_ptr(yp, n, dtype, dev)
                y.copy_(torch.as_tensor(apply(x), device=dev).to(dtype).reshape(n))
                return 0
            except Exception as exc:  # reported after the solver returns
                errors.append(exc)
                return -1

        cb = _lib.MATVEC_FN(_cb)
        keep.append(cb)
        fn = _lib._c.cast(cb, _lib._vp)
        ctx = _lib._vp(0)

    eig = _lib._f64()
    nit = _lib._i32()
    res = _lib._f64()
    vec = torch.empty(n, dtype=dtype, device=dev)
    record = log_level <= logging.DEBUG
    if record:
        max_rows = 2 * int(maxiter) + 64
        rows = np.zeros((max_rows, 6), dtype=np.float64)
        count = _lib._i64(0)
        _lib.call('sqd_locg_record', rows.ctypes.data_as(_lib._vp), max_rows,
                  _lib._c.byref(count))
        print('Performing first LOBPCG steps', flush=True)
    status = _lib.load().sqd_locg(
        n, code, fn, ctx, _lib.ptr(xinit_t), xinit_index, orth_arr, len(orth_t),
        -1.0 if tol is None else float(tol), int(maxiter), mode_code, 1 if use_graph else 0,
        _lib.stream_ptr(), _lib._c.byref(eig), _lib.ptr(vec), _lib._c.byref(nit),
        _lib._c.byref(res))
    if not isinstance(mat, SQDOperator) and errors:
        raise errors[0]
    if status != _lib.SQD_OK and record:
        _lib.call('sqd_locg_record', _lib._vp(0), 0, None)
    _lib.check(status)
    ground_locg.last_residual = res.value
    if record:
        ground_locg.last_history = rows[:count.value].copy()
        _print_history(ground_locg.last_history)
    return eig.value, vec, nit.value


def _print_history(rows):
    """The reference's debug lines (ground_locg.py:330-331, 377-378), one iteration each."""
    for phase, it, theta, r, reltol, conv in rows:
        if phase == 1:
            print(f'FP32 sweep {int(it) - 1}', flush=True)
            print(f'Residual {r}, target {reltol}, theta {theta}, converged: {bool(conv)}',
                  flush=True)
        else:
            print(f'LOCG iteration {int(it) - 1}', flush=True)
            print(f'Residual {r}, reltol {reltol}, converged: {bool(conv)}', flush=True)


def _torch_dtype(dt):
    if isinstance(dt, torch.dtype):
        return dt
    dt = np.dtype(dt)
    return {np.dtype(np.float64): torch.float64, np.dtype(np.complex128): torch.complex128,
            np.dtype(np.float32): torch.float64, np.dtype(np.complex64): torch.complex128}[dt]
