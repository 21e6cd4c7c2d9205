r"""Sample-based quantum diagonalization on a B200 (drop-in for ``rqutils.sqd``).

Same entry points and argument meaning as the reference (``sqd``, ``hproj``, ``run_sqd``,
``SQDOptions``, ``uniquify_states``, ``get_xsource``, ``get_diagonal``), with every step on the
GPU through the C ABI of ``libsqd_b200.so``:

* states are packed to uint64 (bit q = qubit q) and sorted/uniquified by a device radix sort;
  ascending uint64 order is the reference's order of padded big-endian byte rows, so basis
  order and eigenvector indexing match the reference exactly;
* the b XOR x source lookups run once per operator over all (row, X-group) pairs with sector
  and bitmap filters and a device hash table (``cache_strategy`` x = 1), or inside every matvec
  (x = 0);
* the matvec composes the diagonals from popcount(s & z) on the fly (z = 0/1) or reads them
  from a cache of the stored pairs (z = 2);
* ``ground_locg`` runs on the device with fused BLAS-1/Gram kernels and a CUDA-graph loop.

Fill-in slots (``states_size`` larger than the number of unique states) are kept as trailing
vector entries exactly as the reference's 255-rows are: they take part in the convergence test's
vector length and carry the same connectivity.
"""
from dataclasses import dataclass, field
import logging
import time
from typing import Any, Optional

import numpy as np
import torch

from . import _lib
from .paulis.symplectic import PauliSumXZ
from .ground_locg import ground_locg

LOG = logging.getLogger(__name__)

_LOOKUPS = {'hash': _lib.SQD_LOOKUP_HASH, 'bsearch': _lib.SQD_LOOKUP_BSEARCH,
            'auto': _lib.SQD_LOOKUP_AUTO, 'product': _lib.SQD_LOOKUP_PRODUCT}


@dataclass(frozen=True)
class SQDOptions:
    """Options of ``sqd`` (sqd.py:183-196) plus B200 extensions (after ``locg_tol``).

    ``cache_strategy`` keeps the reference's meaning for what is cached, with two merges:

    * ``(0, 1)`` and ``(0, 2)`` run as ``(0, 0)``: without cached sources every matvec looks the
      sources up again, and the diagonal of each found pair is recomputed beside that lookup
      from popcounts, so nothing is stored per pair (the reference stores sign bits or diagonals
      for all N rows of every group, sqd.py:106-122).
    * ``(1, 1)`` runs as ``(1, 0)``: the diagonals are recomputed from popcounts per stored pair
      instead of from packed sign bits.  The reference's ``compute_diagonal`` reads the bit of
      term t at ``t & 255`` instead of ``t & 7`` (sqd.py:590), so its (x, 1) results are wrong
      for groups of more than 8 terms; these strategies give the correct diagonal.

    All strategies give the same Hv (to rounding); they differ in memory and speed: ``(1, 2)``
    stores one element per (row, group) pair whose source exists and is the fastest matvec.
    """
    return_eigvec: bool = True
    cache_strategy: tuple[int, int] = (1, 0)
    shard_bundle: int = 1
    locg_maxiter: int = 1000
    locg_tol: float | None = None
    # --- extensions
    lookup: str = 'auto'             # b XOR x search: 'hash', 'bsearch', 'product' or 'auto'
    locg_mode: str = 'fp64'          # 'fp64' (reference algorithm) or 'mixed'
    use_graph: bool = True           # run the LOCG loop as one CUDA graph
    lanes_per_row: Optional[int] = None   # matvec schedule; None = from the mean row length
    autotune: bool = False           # pick lanes_per_row by timing
    # With cache_strategy (1, 0) or (1, 1): cache the elements of the stored pairs, i.e. run
    # as (1, 2), when they fit in a quarter of the free device memory (the same Hv to
    # rounding, several times faster), with the product-subspace layout where it applies.
    # False keeps the requested strategy.
    promote_cache: bool = True


class Subspace:
    """Sorted, de-duplicated subspace on the GPU (uniquify_states, sqd.py:445-482)."""

    def __init__(self, handle, num_qubits, device):
        self._handle = handle
        self.num_qubits = num_qubits
        self.device = device
        nu, size, nsec = _lib._i64(), _lib._i64(), _lib._i32()
        masks = (_lib._u64 * 2)()
        _lib.call('sqd_space_info', handle, _lib._c.byref(nu), _lib._c.byref(size),
                  _lib._c.byref(nsec), masks)
        self.n_unique = nu.value
        self.states_size = size.value
        self.num_sectors = nsec.value
        self.sector_masks = (masks[0], masks[1])

    @classmethod
    def from_u64(cls, states, num_qubits, states_size=None):
        """``states``: uint64 values (torch int64 tensor or numpy uint64 array)."""
        _lib.require_cuda()
        dev = torch.device('cuda', torch.cuda.current_device())
        if isinstance(states, np.ndarray):
            states = torch.as_tensor(np.ascontiguousarray(states.astype(np.uint64)).view(np.int64))
        states = states.to(dev).contiguous()
        n_in = states.shape[0]
        size = n_in if states_size is None else int(states_size)
        h = _lib._vp()
        _lib.call('sqd_space_create', _lib.ptr(states), n_in, num_qubits, size,
                  _lib.stream_ptr(), _lib._c.byref(h))
        return cls(h, num_qubits, dev)

    @classmethod
    def from_bits(cls, states, states_size=None):
        """Binary [N, n] states in Qiskit order (last column = qubit 0), as in ``sqd``."""
        _lib.require_cuda()
        dev = torch.device('cuda', torch.cuda.current_device())
        bits = torch.as_tensor(np.ascontiguousarray(np.asarray(states).astype(np.uint8)))
        n_in, nq = bits.shape
        bits = bits.to(dev)
        packed = torch.empty(n_in, dtype=torch.int64, device=dev)
        _lib.call('sqd_pack_states', _lib.ptr(bits), n_in, nq, _lib.ptr(packed),
                  _lib.stream_ptr())
        return cls.from_u64(packed, nq, states_size)

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                _lib.load().sqd_space_destroy(h)
            except Exception:  # pragma: no cover
                pass

    @property
    def handle(self):
        return self._handle

    def states(self):
        """Sorted unique states as an int64 CUDA tensor holding the uint64 bit patterns."""
        out = torch.empty(self.n_unique, dtype=torch.int64, device=self.device)
        _lib.call('sqd_space_states', self._handle, _lib.ptr(out), _lib.stream_ptr())
        return out

    def states_bits(self):
        """Unique states as a binary [n_unique, n] uint8 array (Qiskit order)."""
        vals = self.states().cpu().numpy().view(np.uint64)
        n = self.num_qubits
        shifts = np.arange(n - 1, -1, -1, dtype=np.uint64)
        return ((vals[:, None] >> shifts[None, :]) & np.uint64(1)).astype(np.uint8)

    def xsource(self, x, lookup='hash'):
        """get_xsource for one X mask (uint64): int32 CUDA tensor of states_size entries."""
        out = torch.empty(self.states_size, dtype=torch.int32, device=self.device)
        _lib.call('sqd_xsource', self._handle, _lib._u64(int(x)), _LOOKUPS[lookup],
                  _lib.ptr(out), _lib.stream_ptr())
        return out

    def lookup(self, keys, lookup='hash'):
        """Sorted index of each key (int64 CUDA tensor of uint64 bit patterns), -1 when the
        key is not a state of the subspace: int32 CUDA tensor."""
        keys = keys.to(self.device, torch.int64).contiguous()
        out = torch.empty(keys.shape[0], dtype=torch.int32, device=self.device)
        _lib.call('sqd_space_lookup', self._handle, _lib.ptr(keys), keys.shape[0],
                  _LOOKUPS[lookup], _lib.ptr(out), _lib.stream_ptr())
        return out


class SQDOperator:
    """The Hamiltonian projected on a subspace; callable as ``op(v) -> Hv``."""

    def __init__(self, hamiltonian, space, cache_strategy=(1, 0), lookup='auto',
                 lanes_per_row=None):
        self.hamiltonian = hamiltonian
        self.space = space
        x_cache, z_cache = (int(v) for v in cache_strategy)
        h = _lib._vp()
        _lib.call('sqd_op_create', hamiltonian.handle, space.handle, x_cache, z_cache,
                  _LOOKUPS[lookup], _lib.stream_ptr(), _lib._c.byref(h))
        self._handle = h
        nnz, size, cpx = _lib._i64(), _lib._i64(), _lib._i32()
        _lib.call('sqd_op_info', h, _lib._c.byref(nnz), _lib._c.byref(size), _lib._c.byref(cpx))
        self.nnz = nnz.value
        self.size = size.value
        self.value_complex = bool(cpx.value)
        self.cache_strategy = (x_cache, z_cache)
        if lanes_per_row is not None:
            self.lanes_per_row = lanes_per_row

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                _lib.load().sqd_op_destroy(h)
            except Exception:  # pragma: no cover
                pass

    @property
    def handle(self):
        return self._handle

    @property
    def dtype(self):
        """Vector dtype of the reference (vspace dtype = c.dtype, sqd.py:433)."""
        return torch.complex128 if self.value_complex else torch.float64

    @property
    def lanes_per_row(self):
        """Lanes per row of the FP64-vector matvec (the FP32 one: ``get_lanes(1)``)."""
        return self.get_lanes(0)

    @lanes_per_row.setter
    def lanes_per_row(self, v):
        self.set_lanes(0, v)
        self.set_lanes(1, v)

    def get_lanes(self, precision):
        v = _lib._i32()
        _lib.call('sqd_op_get_lanes', self._handle, int(precision), _lib._c.byref(v))
        return v.value

    def set_chunk(self, precision, chunk_rows):
        """Rows a thread block owns at a time in the cached matvec (0 = interleaved)."""
        _lib.call('sqd_op_set_chunk', self._handle, int(precision), int(chunk_rows))
        self._chunk = getattr(self, '_chunk', [0, 0])
        self._chunk[precision] = int(chunk_rows)

    def get_chunk(self, precision):
        return getattr(self, '_chunk', [0, 0])[precision]

    def set_lanes(self, precision, lanes):
        """precision 0: FP64 vectors (float64/complex128), 1: FP32 vectors."""
        _lib.call('sqd_op_set_lanes', self._handle, int(precision), int(lanes))

    LAYOUTS = {'csr': 0, 'product': 1, 'product-csr': 2}

    def set_layout(self, precision, layout):
        """Element layout of the cached matvec for one precision: 'csr' (one pair list per
        row), 'product' (dense slabs for the pairs that change one half of the qubits; the
        other pairs gather from shared memory when their source slabs fit there) or
        'product-csr' (the same slabs, the other pairs always on CSR lists).  The product
        layouts need a product subspace and are built on first use."""
        _lib.call('sqd_op_set_layout', self._handle, int(precision), self.LAYOUTS[layout],
                  _lib.stream_ptr())

    def get_layout(self, precision):
        v = _lib._i32()
        _lib.call('sqd_op_get_layout', self._handle, int(precision), _lib._c.byref(v))
        return {k: n for n, k in self.LAYOUTS.items()}[v.value]

    def product_info(self):
        """{'n_high', 'n_low', 'pairs_high', 'pairs_low', 'pairs_mixed'}; n_high = n_low = 0
        when the subspace is not a product, pair counts -1 until the slabs are built."""
        vals = [_lib._i64() for _ in range(5)]
        _lib.call('sqd_op_product_info', self._handle, _lib.stream_ptr(),
                  *[_lib._c.byref(v) for v in vals])
        keys = ('n_high', 'n_low', 'pairs_high', 'pairs_low', 'pairs_mixed')
        return dict(zip(keys, (v.value for v in vals)))

    @property
    def has_product_layout(self):
        """True when the product layout applies (cached elements, product subspace)."""
        if tuple(self.cache_strategy) != (1, 2):
            return False
        return self.product_info()['n_high'] > 0

    def matvec(self, v, out=None):
        v = v.contiguous()
        if v.shape[0] != self.size:
            raise ValueError(f'vector length {v.shape[0]} != operator size {self.size}')
        if out is None:
            out = torch.empty_like(v)
        _lib.call('sqd_matvec', self._handle, _lib.ptr(v), _lib.ptr(out),
                  _lib.dtype_code(v.dtype), _lib.stream_ptr())
        return out

    __call__ = matvec

    def diagonal(self, group=0, dtype=None):
        dtype = dtype or self.dtype
        out = torch.empty(self.size, dtype=dtype, device=self.space.device)
        _lib.call('sqd_diagonal', self._handle, int(group), _lib.ptr(out),
                  _lib.dtype_code(dtype), _lib.stream_ptr())
        return out

    def vinit(self):
        idx = _lib._i64()
        _lib.call('sqd_vinit', self._handle, _lib._c.byref(idx), _lib.stream_ptr())
        return idx.value

    def csr(self):
        """(indptr int64, indices int32, data complex128) CUDA tensors of <i|H|j>."""
        dev = self.space.device
        indptr = torch.empty(self.size + 1, dtype=torch.int64, device=dev)
        indices = torch.empty(max(self.nnz, 1), dtype=torch.int32, device=dev)[:self.nnz]
        data = torch.empty(max(self.nnz, 1), dtype=torch.complex128, device=dev)[:self.nnz]
        _lib.call('sqd_op_csr', self._handle, _lib.ptr(indptr), _lib.ptr(indices),
                  _lib.ptr(data), _lib.stream_ptr())
        return indptr, indices, data

    def cache_values(self):
        """Cache the element of every stored pair: cache_strategy (1, 0)/(1, 1) -> (1, 2)."""
        _lib.call('sqd_op_cache_values', self._handle, _lib.stream_ptr())
        self.cache_strategy = (1, 2)

    def element_bytes(self):
        """Device bytes the cached elements take with their FP32 copy and, on a product
        subspace, the slab copies of both precisions (an upper bound)."""
        per = 16 if self.value_complex else 8
        return int(self.nnz * per * 3)

    def promote_cache(self, fraction=0.25):
        """(1, 0)/(1, 1) -> (1, 2) when ``element_bytes()`` fits in ``fraction`` of the free
        device memory; the product layout is selected when the subspace is a product of
        high-half and low-half strings.  Returns True when the elements were cached."""
        if tuple(self.cache_strategy) == (1, 2):
            return True
        if self.cache_strategy[0] != 1:
            return False
        free, _ = torch.cuda.mem_get_info(self.space.device)
        if self.element_bytes() > fraction * free:
            return False
        self.cache_values()
        if self.has_product_layout:
            self.set_layout(0, 'product')
            self.set_layout(1, 'product')
        return True

    def refresh(self):
        """Recompute the cached matrix elements after ``hamiltonian.set_coeffs``."""
        _lib.call('sqd_op_refresh', self._handle, _lib.stream_ptr())

    def grad_terms(self, u, v):
        """Re <u|P_t|v> for every merged term t (FP64 CUDA tensor of num_terms)."""
        out = torch.empty(self.hamiltonian.num_terms, dtype=torch.float64,
                          device=self.space.device)
        dt = torch.complex128 if (u.is_complex() or v.is_complex() or self.value_complex) \
            else torch.float64
        u = u.to(dt).contiguous()
        v = v.to(dt).contiguous()
        _lib.call('sqd_grad_terms', self._handle, _lib.ptr(u), _lib.ptr(v),
                  _lib.dtype_code(dt), _lib.ptr(out), _lib.stream_ptr())
        return out

    def autotune(self, dtype=None, candidates=(2, 4, 8, 16, 32), reps=5, **kw):
        """Times the matvec for every schedule (layout, lanes per row, chunk rows) and keeps
        the fastest, for the precision of ``dtype`` (both precisions when ``dtype`` is None).
        Extra keywords go to ``autotune.tune_lanes`` (``chunks``, ``layouts``)."""
        from .autotune import tune_lanes
        if dtype is not None:
            return tune_lanes(self, dtype, candidates, reps, **kw)
        return {'fp64': tune_lanes(self, torch.complex128, candidates, reps, **kw),
                'fp32': tune_lanes(self, torch.complex64, candidates, reps, **kw)}


def _as_pauli(hamiltonian):
    if isinstance(hamiltonian, PauliSumXZ):
        return hamiltonian
    return PauliSumXZ.from_paulisum(hamiltonian, force_real=True, add_padding=True)


def sqd(hamiltonian, states, states_size=None, options=None):
    """Sample-based quantum diagonalization (sqd.py:199-266).

    Returns the ground energy, or (energy, eigenvector[dim] as numpy, basis states uint8
    [dim, n]) if ``options.return_eigvec``.
    """
    if isinstance(options, dict):
        options = SQDOptions(**options)
    if options is None:
        options = SQDOptions()
    states = np.asarray(states)
    if states_size is None:
        states_size = states.shape[0]
    if states_size < states.shape[0]:
        raise ValueError('states_size smaller than the states array length')
    hamiltonian = _as_pauli(hamiltonian)
    LOG.debug('Starting SQD with array size %s', states_size)
    start = time.time()
    result = run_sqd(hamiltonian, states, states_size, options)
    LOG.info('Found ground eigenpair in %f seconds.', time.time() - start)
    eigval = float(result[0])
    if options.return_eigvec:
        eigvec, space, subspace_dim = result[1:]
        basis_states = space.states_bits()[:subspace_dim, -states.shape[1]:]
        return eigval, eigvec[:subspace_dim].cpu().numpy(), basis_states
    return eigval


def run_sqd(hamiltonian, states, states_size, options=None, log_level=logging.INFO):
    """run_sqd (sqd.py:317-442).  ``states``: binary [N, n] array, or a ``Subspace``.
    Returns (eigval,) or (eigval, eigvec, space, subspace_dim).

    ``log_level <= logging.DEBUG`` prints the reference's progress lines (sqd.py:338-430) and
    the solver's per-iteration lines.  (The reference's own ``jax.debug.print(ordered=True)(...)``
    calls there pass no format string to ``jax.debug.print`` and raise at that level.)"""
    if options is None:
        options = SQDOptions()
    debug = log_level <= logging.DEBUG
    hamiltonian = _as_pauli(hamiltonian)
    if debug:
        print(f'Uniquifying states (size {states_size})', flush=True)
    space = states if isinstance(states, Subspace) else Subspace.from_bits(states, states_size)
    if debug and options.cache_strategy[0] > 0:
        print('Precomputing xsources', flush=True)
    if debug and options.cache_strategy == (1, 2):
        print('Precomputing diagonals', flush=True)
    op = SQDOperator(hamiltonian, space, options.cache_strategy, options.lookup,
                     options.lanes_per_row)
    if options.promote_cache and tuple(options.cache_strategy) in ((1, 0), (1, 1)):
        op.promote_cache()
    if options.autotune and options.lanes_per_row is None:
        op.autotune()
    if debug:
        print('Generating vinit', flush=True)
    vinit = op.vinit()
    if debug:
        print(f'Starting minimization with cache_strategy {tuple(options.cache_strategy)}',
              flush=True)
    eigval, eigvec, _ = ground_locg(op, vinit, maxiter=options.locg_maxiter,
                                    tol=options.locg_tol, vspace=(space.states_size, op.dtype),
                                    log_level=log_level, mode=options.locg_mode,
                                    use_graph=options.use_graph)
    result = (eigval,)
    if options.return_eigvec:
        result += (eigvec, space, space.n_unique)
    return result


def _packed_rows(states_p):
    """The reference's packed state rows (sqd.py:255: pad bit, then the qubits, big-endian;
    uint8 [N, B]) as big-endian row values: (int64 CUDA tensor, B, fill-row mask).  Rows of 255
    are the reference's fill rows; any other row with the pad bit set is rejected."""
    _lib.require_cuda()
    dev = torch.device('cuda', torch.cuda.current_device())
    t = states_p if isinstance(states_p, torch.Tensor) else torch.as_tensor(np.asarray(states_p))
    if t.dtype != torch.uint8 or t.dim() != 2:
        raise ValueError('packed states must be a uint8 array of shape [N, B]')
    b = t.shape[1]
    if not 1 <= b <= 8:
        raise ValueError('packed rows of 1 to 8 bytes (up to 63 qubits) are supported')
    t = t.to(dev)
    keys = torch.zeros(t.shape[0], dtype=torch.int64, device=dev)
    for c in range(b):
        keys = (keys << 8) | t[:, c].to(torch.int64)
    fill = (t == 255).all(dim=1)
    if bool(((t[:, 0] >= 128) & ~fill).any()):
        raise ValueError('a packed state row has the pad bit set but is not a fill row of 255')
    return keys, b, fill


def _host_array(a):
    return a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else a


def _packed_x(xsignature, b):
    x = np.asarray(_host_array(xsignature), dtype=np.uint8).reshape(-1)
    if x.shape[0] != b:
        raise ValueError(f'xsignature has {x.shape[0]} bytes, the states {b}')
    if x[0] >= 128:
        raise ValueError('xsignature has the pad bit set')
    return int.from_bytes(x.tobytes(), 'big')


def uniquify_states(states_p, states_size, return_indices=False):
    """uniquify_states (sqd.py:445-482) on the reference's packed rows (uint8 [N, B]): the sorted
    unique rows followed by rows of 255 up to ``states_size`` (a uint8 CUDA tensor), and with
    ``return_indices`` the input index of each kept row (its last occurrence, as the reference's
    stable sort gives; -1 for fill rows).  Sorting and de-duplication run on the device
    (``Subspace``); ``Subspace.from_bits`` takes binary states instead.  As in the reference, a
    ``states_size`` below the number of unique rows keeps the first ``states_size`` of them."""
    keys, b, fill = _packed_rows(states_p)
    dev = keys.device
    states_size = int(states_size)
    real_idx = torch.nonzero(~fill).flatten()
    real = keys[real_idx]
    out = torch.full((states_size, b), 255, dtype=torch.uint8, device=dev)
    idx = torch.full((states_size,), -1, dtype=torch.int32, device=dev)
    n_u = 0
    if real.numel():
        space = Subspace.from_u64(real, 8 * b - 1)
        uniq = space.states()
        n_u = uniq.numel()
        m = min(n_u, states_size)
        for c in range(b):
            out[:m, c] = ((uniq[:m] >> (8 * (b - 1 - c))) & 255).to(torch.uint8)
        if return_indices:
            pos = space.lookup(real).long()
            last = torch.full((n_u,), -1, dtype=torch.int64, device=dev)
            last.scatter_reduce_(0, pos, real_idx, reduce='amax')
            idx[:m] = last[:m].to(torch.int32)
    if return_indices and bool(fill.any()) and n_u < states_size:
        idx[n_u] = int(torch.nonzero(fill).max())   # the rows of 255 sort last
    return (out, idx) if return_indices else out


def get_xsource(xsignature, states, sorted_input=True, lookup='hash'):
    """get_xsource (sqd.py:485-548): int32 CUDA tensor, entry i the index of the row equal to
    row i XOR x, or -1.

    ``states`` is a ``Subspace`` (x: uint64 or packed bytes) or, as in the reference, packed rows
    (uint8 [N, B], x: B packed bytes).  With ``sorted_input=True`` the rows must be sorted and
    unique, optionally followed by fill rows of 255 (the output of ``uniquify_states``); the fill
    rows get the values the reference's sort-based algorithm gives them.  With
    ``sorted_input=False`` the rows may come in any order (sqd.py:515-516, 542-545) and indices
    refer to the input order; duplicate rows and fill rows are rejected there, because the
    reference's scatter then writes one position several times (its result is undefined)."""
    xsignature = _host_array(xsignature)
    if isinstance(states, Subspace):
        if isinstance(xsignature, (np.ndarray, list, tuple)):
            from .paulis.symplectic import _unpack_masks
            xsignature = int(_unpack_masks(np.asarray(xsignature, dtype=np.uint8)[None, :],
                                           states.num_qubits, True)[0])
        return states.xsource(int(xsignature), lookup)
    keys, b, fill = _packed_rows(states)
    x = _packed_x(xsignature, b)
    n = keys.shape[0]
    dev = keys.device
    if n == 0:
        return torch.empty(0, dtype=torch.int32, device=dev)
    nq = 8 * b - 1
    if sorted_input:
        n_real = int((~fill).sum())
        ok = bool((~fill[:n_real]).all()) and bool(fill[n_real:].all()) and n_real > 0
        ok = ok and bool((keys[1:n_real] > keys[:n_real - 1]).all())
        if not ok:
            raise ValueError('sorted_input=True needs sorted unique rows followed by fill rows '
                             'of 255 (the output of uniquify_states); pass sorted_input=False')
        return Subspace.from_u64(keys[:n_real], nq, states_size=n).xsource(x, lookup)
    if bool(fill.any()):
        raise ValueError('fill rows of 255 with sorted_input=False: the reference scatters them '
                         'all to one position')
    space = Subspace.from_u64(keys, nq)
    if space.n_unique != n:
        raise ValueError('duplicate rows with sorted_input=False: the reference scatters them '
                         'to one position')
    pos = space.lookup(keys).long()
    inv = torch.empty(n, dtype=torch.int64, device=dev)
    inv[pos] = torch.arange(n, dtype=torch.int64, device=dev)
    src = space.lookup(keys ^ x, lookup).long()
    return torch.where(src >= 0, inv[src.clamp(min=0)], torch.full_like(src, -1)).to(torch.int32)


def get_diagonal(op, group):
    """get_diagonal (sqd.py:603-628) of group ``group`` for every slot of the operator."""
    return op.diagonal(group)


def hproj(hamiltonian, states, unique_states=False):
    """Projected Hamiltonian as a scipy CSR matrix (sqd.py:269-314).  The states are packed
    consistently with the padded Hamiltonian (the reference packs them without the pad bit,
    sqd.py:298, so its byte widths disagree)."""
    from scipy.sparse import csr_array
    if not isinstance(hamiltonian, PauliSumXZ):
        hamiltonian = PauliSumXZ.from_paulisum(hamiltonian, add_padding=True)
    states = np.asarray(states)
    space = Subspace.from_bits(states)
    op = SQDOperator(hamiltonian, space, cache_strategy=(1, 0))
    indptr, indices, data = (t.cpu().numpy() for t in op.csr())
    if not hamiltonian.is_complex:
        data = data.real
    n = space.n_unique
    return csr_array((data, indices, indptr[:n + 1]), shape=(n, n))
