"""Many SQD instances solved together on one GPU.

``SQDBatch`` concatenates operators with cached matrix elements (cache_strategy (1, 2)) into one
block-diagonal operator and runs the batched mixed-precision LOCG (``sqd_batch_locg``): one
tile work queue over all instances' rows that skips converged instances, per-instance
reductions and Rayleigh-Ritz steps, the iteration loop as one CUDA graph.  ``solve_instances``
schedules a list of problems in waves that fit a device-memory budget; instances too large to
share a wave are solved alone with the single-instance mixed solver.
"""
import numpy as np
import torch

from . import _lib
from .paulis.symplectic import PauliSumXZ
from .sqd import SQDOperator, Subspace
from .ground_locg import ground_locg


class SQDBatch:
    def __init__(self, ops):
        if not ops:
            raise ValueError('no operators')
        arr = (_lib._vp * len(ops))(*[op.handle.value for op in ops])
        h = _lib._vp()
        _lib.call('sqd_batch_create', arr, len(ops), _lib.stream_ptr(), _lib._c.byref(h))
        self._handle = h
        self.sizes = [op.size for op in ops]
        self.value_complex = ops[0].value_complex
        rows, pairs = _lib._i64(), _lib._i64()
        _lib.call('sqd_batch_info', h, _lib._c.byref(rows), _lib._c.byref(pairs))
        self.total_rows, self.total_pairs = rows.value, pairs.value
        self.device = ops[0].space.device

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                _lib.load().sqd_batch_destroy(h)
            except Exception:  # pragma: no cover
                pass

    def set_lanes(self, precision, lanes):
        _lib.call('sqd_batch_set_lanes', self._handle, int(precision), int(lanes))

    def solve(self, xinit_index=None, xinit=None, tol=None, maxiter=1000, use_graph=True,
              dtype=None):
        """Returns (eigvals[n], eigvecs list of CUDA tensors, niters[n], residuals[n])."""
        n = len(self.sizes)
        dtype = dtype or (torch.complex128 if self.value_complex else torch.float64)
        idx = None
        x0 = None
        if xinit is not None:
            x0 = torch.cat([torch.as_tensor(v, device=self.device).to(dtype) for v in xinit])
        else:
            if xinit_index is None:
                raise ValueError('xinit or xinit_index is required')
            idx = (_lib._i64 * n)(*[int(i) for i in xinit_index])
        eig = (_lib._f64 * n)()
        nit = (_lib._i32 * n)()
        res = (_lib._f64 * n)()
        vecs = torch.empty(self.total_rows, dtype=dtype, device=self.device)
        _lib.call('sqd_batch_locg', self._handle, _lib.dtype_code(dtype), _lib.ptr(x0), idx,
                  -1.0 if tol is None else float(tol), int(maxiter), 1 if use_graph else 0,
                  _lib.stream_ptr(), eig, _lib.ptr(vecs), nit, res)
        out, off = [], 0
        for s in self.sizes:
            out.append(vecs[off:off + s])
            off += s
        return np.array(eig[:]), out, np.array(nit[:]), np.array(res[:])


def _operator(inst):
    ham = PauliSumXZ.from_xz(inst.x, inst.z, inst.coeffs, inst.num_qubits, force_real=True,
                             padded=True)
    space = Subspace.from_u64(inst.states, inst.num_qubits)
    return SQDOperator(ham, space, cache_strategy=(1, 2))


def solve_instances(instances, budget_bytes=48 << 30, alone_pairs=int(1.5e9), tol=None,
                    maxiter=1000, use_graph=True, dtype=torch.complex128):
    """Ground energies of many SQD problems (objects with x, z, coeffs, num_qubits, states),
    started from each problem's vinit.  Returns (eigvals, niters) in input order."""
    n = len(instances)
    eig = np.zeros(n)
    nit = np.zeros(n, dtype=np.int64)
    wave, wave_ops, wave_bytes = [], [], 0

    def flush():
        nonlocal wave, wave_ops, wave_bytes
        if not wave:
            return
        starts = [op.vinit() for op in wave_ops]
        batch = SQDBatch(wave_ops)
        wave_ops.clear()          # the batch holds copies; the operators are freed here
        e, _, it, _ = batch.solve(xinit_index=starts, tol=tol, maxiter=maxiter,
                                  use_graph=use_graph, dtype=dtype)
        eig[wave] = e
        nit[wave] = it
        del batch
        wave, wave_bytes = [], 0

    for i, inst in enumerate(instances):
        op = _operator(inst)
        if op.nnz > alone_pairs:
            _lib.call('sqd_op_release_groups', op.handle)
            x0 = op.vinit()
            e, _, it = ground_locg(op, x0, tol=tol, maxiter=maxiter, mode='mixed',
                                   use_graph=use_graph, vspace=(op.size, dtype))
            eig[i], nit[i] = e, it
            del op
            # The library pool keeps the freed memory for the next wave's tables; return it to
            # the driver only when little is left for other allocators (torch's vectors).
            free, _ = torch.cuda.mem_get_info()
            if free < (8 << 30):
                _lib.trim_memory()
            continue
        need = op.nnz * 16 + op.size * 7 * 16
        if wave and wave_bytes + need > budget_bytes:
            flush()
        wave.append(i)
        wave_ops.append(op)
        wave_bytes += need
    flush()
    return eig, nit
