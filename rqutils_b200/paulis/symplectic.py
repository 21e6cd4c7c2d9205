r"""Symplectic (XZ) Pauli sums resident on a B200 (drop-in for ``rqutils.paulis.symplectic``).

A Pauli string is :math:`Q = (-i)^{x \cdot z} Z^{z} X^{x}` with bit masks ``x`` and ``z``
(bit q = qubit q; a label's character 0 is qubit n-1).  ``PauliSumXZ.from_paulisum`` groups the
terms by X mask on the GPU (device-side sort, merge, grouping and phase multiplication in
``csrc/paulis.cu``); the grouped table stays on the device as CSR arrays.  The reference's
byte-packed fields ``x``, ``z``, ``c`` (paulis/symplectic.py:41-48) are produced on demand for
compatibility.
"""
import warnings

import numpy as np
import torch

from .. import _lib
from ..workloads import xz_from_labels

try:  # optional input type, as in the reference (symplectic.py:34-38)
    from qiskit.quantum_info import SparsePauliOp
    HAS_QISKIT = True
except ImportError:  # pragma: no cover - qiskit is not installed in this image
    HAS_QISKIT = False


class PauliSumXZ:
    """Symplectic representation of a sum of Pauli strings (symplectic.py:41-149).

    Construct with :meth:`from_paulisum`, :meth:`from_xz`, or — like the reference dataclass —
    from byte-packed arrays ``PauliSumXZ(x, z, c, num_qubits)``.
    """

    def __init__(self, x=None, z=None, c=None, num_qubits=None, *, padded=True, _handle=None,
                 _meta=None):
        self._handle = None
        self._device = None
        self._padded = padded
        self._cache = {}
        if _handle is not None:
            self._handle = _handle
            self._device = torch.device('cuda', torch.cuda.current_device())
            self.num_qubits = num_qubits
            self._meta = _meta
            return
        if x is None or z is None or c is None or num_qubits is None:
            raise ValueError('PauliSumXZ needs x, z, c and num_qubits')
        # Byte-packed reference layout -> raw terms (one per stored slot up to the first zero
        # coefficient of each group, which is where the reference's get_diagonal stops).
        x = np.asarray(x, dtype=np.uint8)
        z = np.asarray(z, dtype=np.uint8)
        c = np.asarray(c)
        xs, zs, cs = [], [], []
        xm = _unpack_masks(x, num_qubits, padded)
        zm = _unpack_masks(z.reshape(-1, z.shape[-1]), num_qubits, padded).reshape(z.shape[:2])
        for j in range(x.shape[0]):
            for k in range(c.shape[1]):
                if c[j, k] == 0:
                    break
                ph = int(np.bitwise_count(xm[j] & zm[j, k])) & 3
                # stored c = alpha (-i)^ph  ->  alpha = c i^ph
                cs.append(complex(c[j, k]) * (1j ** ph))
                xs.append(xm[j])
                zs.append(zm[j, k])
        other = PauliSumXZ.from_xz(np.array(xs, dtype=np.uint64), np.array(zs, dtype=np.uint64),
                                   np.array(cs), num_qubits, padded=padded)
        self.__dict__.update(other.__dict__)
        other._handle = None

    # ------------------------------------------------------------------ construction
    @classmethod
    def from_paulisum(cls, paulisum, force_real=False, add_padding=False):
        """``PauliSumXZ.from_paulisum`` (symplectic.py:50-124): ``([labels], [coeffs])`` or a
        Qiskit ``SparsePauliOp``."""
        if isinstance(paulisum, tuple):
            paulis, coeffs = paulisum
            if len(paulis) != len(coeffs):
                raise ValueError('Lengths of Pauli and coeff lists do not match')
            if len(set(len(p) for p in paulis)) != 1:
                raise ValueError('Pauli strings have non-uniform lengths')
            x, z, n = xz_from_labels(list(paulis))
            coeffs = np.asarray(coeffs)
        elif HAS_QISKIT and isinstance(paulisum, SparsePauliOp):  # pragma: no cover
            if not np.allclose(paulisum.coeffs.imag, 0.):
                raise ValueError('Coefficients of Paulis must be real for the Hamiltonian to be'
                                 ' Hermitian.')
            paulisum = paulisum.simplify()
            n = paulisum.num_qubits
            w = np.uint64(1) << np.arange(n, dtype=np.uint64)
            x = (paulisum.paulis.x.astype(np.uint64) * w).sum(axis=1, dtype=np.uint64)
            z = (paulisum.paulis.z.astype(np.uint64) * w).sum(axis=1, dtype=np.uint64)
            coeffs = paulisum.coeffs
        else:
            raise ValueError('Unsupported input type')
        return cls.from_xz(x, z, coeffs, n, force_real=force_real, padded=add_padding)

    @classmethod
    def from_xz(cls, x, z, coeffs, num_qubits, force_real=False, padded=False):
        """Raw terms as uint64 X/Z masks plus coefficients (extension of the reference API)."""
        _lib.require_cuda()
        if num_qubits < 1 or num_qubits > 63:
            raise ValueError('num_qubits must be in [1, 63]')
        dev = torch.device('cuda', torch.cuda.current_device())
        x = torch.as_tensor(np.ascontiguousarray(np.asarray(x, dtype=np.uint64)).view(np.int64))
        z = torch.as_tensor(np.ascontiguousarray(np.asarray(z, dtype=np.uint64)).view(np.int64))
        coeffs = np.asarray(coeffs)
        if x.shape[0] != coeffs.shape[0] or z.shape[0] != coeffs.shape[0]:
            raise ValueError('Lengths of Pauli and coeff lists do not match')
        re = torch.as_tensor(np.ascontiguousarray(coeffs.real, dtype=np.float64)).to(dev)
        im = None
        if np.iscomplexobj(coeffs):
            im = torch.as_tensor(np.ascontiguousarray(coeffs.imag, dtype=np.float64)).to(dev)
        x = x.to(dev)
        z = z.to(dev)
        handle = _lib._vp()
        dropped = _lib._c.c_int(0)
        flags = _lib.SQD_PAULIS_FORCE_REAL if force_real else 0
        _lib.call('sqd_paulis_create', _lib.ptr(x), _lib.ptr(z), _lib.ptr(re), _lib.ptr(im),
                  x.shape[0], num_qubits, flags, _lib.stream_ptr(), _lib._c.byref(handle),
                  _lib._c.byref(dropped))
        if dropped.value:
            warnings.warn('Found nonzero imaginary part when force_real=True')
        meta = _info(handle)
        obj = cls(num_qubits=num_qubits, padded=padded, _handle=handle, _meta=meta)
        obj._num_raw = x.shape[0]
        return obj

    def set_coeffs(self, coeffs):
        """New coefficients for the raw terms this sum was created from (same order); the
        grouping is kept.  Operators built on this sum need ``SQDOperator.refresh()``."""
        coeffs = torch.as_tensor(coeffs)
        if coeffs.shape[0] != self._num_raw:
            raise ValueError('Lengths of Pauli and coeff lists do not match')
        re = coeffs.real if coeffs.is_complex() else coeffs
        re = re.to(device=self._device, dtype=torch.float64).contiguous()
        im = None
        if coeffs.is_complex():
            im = coeffs.imag.to(device=self._device, dtype=torch.float64).contiguous()
        dropped = _lib._c.c_int(0)
        _lib.call('sqd_paulis_set_coeffs', self._handle, _lib.ptr(re), _lib.ptr(im),
                  _lib.stream_ptr(), _lib._c.byref(dropped))
        if dropped.value:
            warnings.warn('Found nonzero imaginary part when force_real=True')
        self._cache.pop('tables', None)
        self._cache.pop('ref', None)

    def raw_to_term(self):
        """int64 CUDA tensor: merged-term index of every raw term (-1 if dropped)."""
        return self.device_tables()[4].to(torch.int64)

    def __del__(self):
        h = getattr(self, '_handle', None)
        if h is not None and h.value:
            try:
                _lib.load().sqd_paulis_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass

    # ------------------------------------------------------------------ properties
    @property
    def handle(self):
        return self._handle

    @property
    def num_groups(self):
        return self._meta['num_groups']

    @property
    def num_terms(self):
        return self._meta['num_terms']

    @property
    def is_complex(self):
        return bool(self._meta['is_complex'])

    def device_tables(self):
        """(group_x, group_start, term_z, term_c, raw_to_term) as CUDA tensors."""
        if 'tables' not in self._cache:
            J, M = self.num_groups, self.num_terms
            d = self._device
            gx = torch.empty(J, dtype=torch.int64, device=d)
            gs = torch.empty(J + 1, dtype=torch.int64, device=d)
            tz = torch.empty(M, dtype=torch.int64, device=d)
            tc = torch.empty(M, dtype=torch.complex128, device=d)
            r2t = torch.empty(self._num_raw, dtype=torch.int32, device=d)
            _lib.call('sqd_paulis_export', self._handle, _lib.ptr(gx), _lib.ptr(gs),
                      _lib.ptr(tz), _lib.ptr(tc), _lib.ptr(r2t), _lib.stream_ptr())
            self._cache['tables'] = (gx, gs, tz, tc, r2t)
        return self._cache['tables']

    def _reference_layout(self):
        if 'ref' not in self._cache:
            gx, gs, tz, tc, _ = (t.cpu().numpy() for t in self.device_tables())
            gx = gx.view(np.uint64)
            tz = tz.view(np.uint64)
            J = gx.shape[0]
            counts = np.diff(gs)
            kmax = int(counts.max())
            n = self.num_qubits
            zfull = np.zeros((J, kmax), dtype=np.uint64)
            cfull = np.zeros((J, kmax), dtype=np.complex128)
            for j in range(J):
                zfull[j, :counts[j]] = tz[gs[j]:gs[j + 1]]
                cfull[j, :counts[j]] = tc[gs[j]:gs[j + 1]]
            if not self.is_complex:
                cfull = cfull.real
            xb = _pack_masks(gx, n, self._padded)
            zb = _pack_masks(zfull.reshape(-1), n, self._padded).reshape(J, kmax, -1)
            self._cache['ref'] = (xb, zb, cfull)
        return self._cache['ref']

    @property
    def x(self):
        """X signatures, uint8 [J, B] big-endian (symplectic.py:45)."""
        return self._reference_layout()[0]

    @property
    def z(self):
        """Z signatures, uint8 [J, K_max, B] (symplectic.py:46)."""
        return self._reference_layout()[1]

    @property
    def c(self):
        """Phased coefficients [J, K_max] (symplectic.py:47)."""
        return self._reference_layout()[2]

    @property
    def arrays(self):
        return self.x, self.z, self.c

    def matmul(self, rhs):
        """H @ rhs on the full 2^n Hilbert space (symplectic.py:130-149), rhs of shape
        [2^n, ...] as a CUDA tensor or an array."""
        from ..sqd import SQDOperator, Subspace
        n = self.num_qubits
        rhs_t = torch.as_tensor(rhs, device=self._device)
        if rhs_t.shape[0] != 2 ** n:
            raise ValueError(f'RHS axis 0 size {rhs_t.shape[0]} is incompatible with'
                             f' num_qubits={n}')
        if 'full_op' not in self._cache:
            states = torch.arange(2 ** n, dtype=torch.int64, device=self._device)
            space = Subspace.from_u64(states, n)
            self._cache['full_op'] = SQDOperator(self, space, cache_strategy=(1, 2))
        op = self._cache['full_op']
        dt = torch.complex128 if (self.is_complex or rhs_t.is_complex()) else torch.float64
        flat = rhs_t.reshape(rhs_t.shape[0], -1).to(dt)
        out = torch.empty_like(flat)
        for k in range(flat.shape[1]):
            out[:, k] = op.matvec(flat[:, k].contiguous())
        return out.reshape((rhs_t.shape[0],) + tuple(rhs_t.shape[1:]))


def _info(handle):
    J = _lib._i64()
    M = _lib._i64()
    K = _lib._i64()
    cpx = _lib._i32()
    nq = _lib._i32()
    _lib.call('sqd_paulis_info', handle, _lib._c.byref(J), _lib._c.byref(M), _lib._c.byref(K),
              _lib._c.byref(cpx), _lib._c.byref(nq))
    return {'num_groups': J.value, 'num_terms': M.value, 'max_k': K.value,
            'is_complex': cpx.value, 'num_qubits': nq.value}


def _pack_masks(masks, n, padded):
    """uint64 masks -> packbits([pad?, b_{n-1}, ..., b_0])."""
    masks = np.asarray(masks, dtype=np.uint64)
    shifts = np.arange(n - 1, -1, -1, dtype=np.uint64)
    bits = ((masks[:, None] >> shifts[None, :]) & np.uint64(1)).astype(np.uint8)
    if padded:
        bits = np.pad(bits, ((0, 0), (1, 0)))
    return np.packbits(bits, axis=-1)


def _unpack_masks(packed, n, padded):
    bits = np.unpackbits(np.asarray(packed, dtype=np.uint8), axis=-1)
    off = 1 if padded else 0
    bits = bits[:, off:off + n].astype(np.uint64)
    weights = np.uint64(1) << np.arange(n - 1, -1, -1, dtype=np.uint64)
    return (bits * weights).sum(axis=1, dtype=np.uint64)
