"""Independent dense oracle (test infrastructure only).

Builds Pauli strings as Kronecker products of 2x2 matrices, with no symplectic bit tricks, in
Qiskit's convention (character 0 of a label is qubit n-1, basis index = sum_q s_q 2^q).  This is
the check the reference's own notebook performs (tests/sqd.ipynb: ``to_matrix()`` projected onto
the unique states, then ``eigh``).
"""
import numpy as np

_PAULI = {
    'I': np.eye(2, dtype=np.complex128),
    'X': np.array([[0, 1], [1, 0]], dtype=np.complex128),
    'Y': np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
    'Z': np.array([[1, 0], [0, -1]], dtype=np.complex128),
}


def pauli_matrix(label):
    mat = np.ones((1, 1), dtype=np.complex128)
    for ch in label.upper():
        mat = np.kron(mat, _PAULI[ch])
    return mat


def hamiltonian_matrix(paulis, coeffs):
    n = len(paulis[0])
    mat = np.zeros((2 ** n, 2 ** n), dtype=np.complex128)
    for label, coeff in zip(paulis, coeffs):
        mat += coeff * pauli_matrix(label)
    return mat


def projected_matrix(paulis, coeffs, indices):
    """<i|H|j> for basis indices (uint64 values) without forming the 2^n matrix: each Pauli
    string is applied to basis vectors through its own single-qubit action."""
    indices = np.asarray(indices, dtype=np.int64)
    n = len(paulis[0])
    pos = {int(v): k for k, v in enumerate(indices)}
    dim = indices.shape[0]
    mat = np.zeros((dim, dim), dtype=np.complex128)
    for label, coeff in zip(paulis, coeffs):
        label = label.upper()
        for col, state in enumerate(indices):
            amp = complex(coeff)
            out = int(state)
            for q in range(n):
                ch = label[n - 1 - q]
                bit = (int(state) >> q) & 1
                if ch == 'X':
                    out ^= (1 << q)
                elif ch == 'Y':
                    out ^= (1 << q)
                    amp *= (1j if bit == 0 else -1j)
                elif ch == 'Z':
                    amp *= (1 if bit == 0 else -1)
            row = pos.get(out)
            if row is not None:
                mat[row, col] += amp
    return mat


def ground_energy(mat):
    vals, vecs = np.linalg.eigh(mat)
    return vals[0], vecs[:, 0]
