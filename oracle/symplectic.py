"""Oracle restatement of ``rqutils/paulis/symplectic.py`` (test infrastructure only).

``from_paulisum`` follows symplectic.py:50-124 (tuple input path); ``matmul`` follows
symplectic.py:130-149.  Arrays keep the reference's byte-packed big-endian layout so that the
restatement can be compared with the reference's documented data structure directly.
"""
import warnings
import numpy as np


class PauliSumXZ:
    """Plain container mirroring ``PauliSumXZ`` (symplectic.py:41-48)."""

    def __init__(self, x, z, c, num_qubits):
        self.x = x
        self.z = z
        self.c = c
        self.num_qubits = num_qubits

    @property
    def arrays(self):
        return self.x, self.z, self.c


def from_paulisum(paulisum, force_real=False, add_padding=False):
    """Restates ``PauliSumXZ.from_paulisum`` (symplectic.py:50-124), tuple path only."""
    if not isinstance(paulisum, tuple):
        raise ValueError('Unsupported input type')
    paulis, coeffs = paulisum
    if len(paulis) != len(coeffs):                         # symplectic.py:59-60
        raise ValueError('Lengths of Pauli and coeff lists do not match')
    if len(set(len(p) for p in paulis)) != 1:              # symplectic.py:61-62
        raise ValueError('Pauli strings have non-uniform lengths')

    coeffs = np.array(coeffs)
    paulis = np.array([list(p.upper()) for p in paulis])    # symplectic.py:66
    nonzero = np.nonzero(coeffs)                            # symplectic.py:67-69
    coeffs = coeffs[nonzero]
    paulis = paulis[nonzero]
    paulis, indices = np.unique(paulis, axis=0, return_inverse=True)   # symplectic.py:70
    indices = indices.reshape(-1)
    # symplectic.py:71-72: merge duplicates with a 0/1 mask matmul
    masks = (indices[None, :] == np.arange(paulis.shape[0])[:, None]).astype(int)
    coeffs = masks @ coeffs
    xbits = np.logical_or(paulis == 'X', paulis == 'Y')     # symplectic.py:73-74
    zbits = np.logical_or(paulis == 'Y', paulis == 'Z')
    num_qubits = paulis.shape[1]

    if force_real:                                          # symplectic.py:92-95
        if np.any(coeffs.imag != 0.):
            warnings.warn('Found nonzero imaginary part when force_real=True')
        coeffs = coeffs.real

    # symplectic.py:98-111: group by X signature, phase (-i)^{popcount(x & z)}
    xuniq, indices, counts = np.unique(xbits, axis=0, return_inverse=True, return_counts=True)
    indices = indices.reshape(-1)
    xsignatures = xuniq.astype(np.uint8)
    shape = (xsignatures.shape[0], np.max(counts))
    zsignatures = np.zeros(shape + zbits.shape[-1:], dtype=np.uint8)
    phcoeffs = np.zeros(shape, dtype=np.complex128)
    for isig, xsig in enumerate(xsignatures):
        ipaulis = np.nonzero(indices == isig)[0]
        zsigs = zbits[ipaulis].astype(np.uint8)
        zsignatures[isig, :counts[isig]] = zsigs
        iphases = np.sum(xsig & zsigs, axis=1) & 3
        phases = np.array([1., -1.j, -1., 1.j])[iphases]
        phcoeffs[isig, :counts[isig]] = coeffs[ipaulis] * phases

    if np.all(phcoeffs.imag == 0.):                         # symplectic.py:113-114
        phcoeffs = phcoeffs.real

    if add_padding:                                         # symplectic.py:116-119
        xsignatures = np.pad(xsignatures, ((0, 0), (1, 0)))
        zsignatures = np.pad(zsignatures, ((0, 0), (0, 0), (1, 0)))

    xsignatures = np.packbits(xsignatures, axis=-1)         # symplectic.py:122-123
    zsignatures = np.packbits(zsignatures, axis=-1)
    return PauliSumXZ(xsignatures, zsignatures, phcoeffs, num_qubits)


def matmul(ham, rhs):
    """Restates ``PauliSumXZ.matmul`` (symplectic.py:130-149): H @ rhs on the full 2^n space.

    ``ham`` must be built without padding.
    """
    if rhs.shape[0] != 2 ** ham.num_qubits:
        raise ValueError(f'RHS axis 0 size {rhs.shape[0]} is incompatible with'
                         f' num_qubits={ham.num_qubits}')
    indices = np.arange(rhs.shape[0], dtype=np.int64)
    nbytes = ham.x.shape[1]
    powers = 256 ** np.arange(nbytes, dtype=np.int64)[::-1]
    offset = 8 * nbytes - ham.num_qubits
    packed_x = np.sum(ham.x.astype(np.int64) * powers, axis=1) >> offset
    packed_z = np.sum(ham.z.astype(np.int64) * powers, axis=2) >> offset
    out = np.zeros(rhs.shape, dtype=np.result_type(rhs.dtype, ham.c.dtype))
    for xsig, zsigs, coeffs in zip(packed_x, packed_z, ham.c):
        signs = 1. - 2. * (np.bitwise_count(indices & zsigs[:, None]) & 1)
        diags = np.sum(coeffs[:, None] * signs, axis=0)
        diags = diags.reshape(diags.shape + (1,) * (rhs.ndim - 1))
        out += rhs[indices ^ xsig] * diags
    return out
