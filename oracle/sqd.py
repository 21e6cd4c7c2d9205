"""Oracle restatement of the SQD path in ``rqutils/sqd.py`` (test infrastructure only).

Byte-packed, padded layout exactly as the reference uses it: a state row is
``packbits([pad, s_{n-1}, ..., s_0])`` with the pad bit 0 for real states and rows of 255 for
fill-in slots.
"""
import numpy as np

from .symplectic import from_paulisum, PauliSumXZ
from .ground_locg import ground_locg


class SQDOptions:
    """Mirror of ``SQDOptions`` (sqd.py:183-196)."""

    def __init__(self, return_eigvec=True, cache_strategy=(1, 0), shard_bundle=1,
                 locg_maxiter=1000, locg_tol=None):
        self.return_eigvec = return_eigvec
        self.cache_strategy = tuple(cache_strategy)
        self.shard_bundle = shard_bundle
        self.locg_maxiter = locg_maxiter
        self.locg_tol = locg_tol


def pack_states(states):
    """sqd.py:255 — pad a leading zero bit and pack big-endian into uint8."""
    return np.packbits(np.pad(np.asarray(states).astype(np.uint8), ((0, 0), (1, 0))), axis=1)


def uniquify_states(states_p, states_size, return_indices=False):
    """Restates ``uniquify_states`` (sqd.py:445-482).

    Lexicographic sort of the packed rows, unique rows kept in sorted order, tail filled with
    rows of 255 up to ``states_size`` (a smaller ``states_size`` keeps the first unique rows:
    the bincount at :465-470 has that length).  The kept position of each unique row is the
    LAST of its run in the stable sort (cumsum of the per-id counts over positions 1..N-1,
    :463-470), so ``return_indices`` gives each row's last input occurrence.
    """
    keys = tuple(states_p[:, b] for b in range(states_p.shape[1] - 1, -1, -1))
    perm = np.lexsort(keys)                                  # stable multi-key sort (:457-458)
    states_srt = states_p[perm]
    is_unique = np.any(states_srt[1:] != states_srt[:-1], axis=1)   # :461
    last = np.concatenate([is_unique, [True]])               # position i ends its run
    uniq = states_srt[last]
    m = min(uniq.shape[0], states_size)
    out = np.full((states_size, states_p.shape[1]), 255, dtype=np.uint8)
    out[:m] = uniq[:m]
    if return_indices:
        idx = np.full(states_size, -1, dtype=np.int64)
        idx[:m] = perm[last][:m]
        return out, idx
    return out


def get_xsource(xsignature, states_p):
    """Restates ``get_xsource`` (sqd.py:485-548) step by step, sorted input.

    Stable sort of the 2N rows [S; S^X] with their indices (:517-523), adjacent equality
    (:526-530) and the cumsum/bincount position map (:533-540).  Fill rows produce exactly the
    values the reference produces for them.
    """
    size = states_p.shape[0]
    mapped = np.bitwise_xor(states_p, xsignature)
    joined = np.concatenate([states_p, mapped], axis=0)
    keys = tuple(joined[:, b] for b in range(joined.shape[1] - 1, -1, -1))
    order = np.lexsort(keys)                                  # stable
    joined_sorted = joined[order]
    idx_sorted = order.astype(np.int64)
    equal = np.all(joined_sorted[:-1] == joined_sorted[1:], axis=1)
    source_idx = np.where(equal, idx_sorted[1:] - size, -1)
    counts = np.bincount(np.cumsum(idx_sorted < size), minlength=size)[:size]
    tposition = np.cumsum(counts)
    out = np.full(size, -1, dtype=np.int64)
    ok = tposition < source_idx.shape[0]
    out[ok] = source_idx[tposition[ok]]
    return out.astype(np.int32)


def get_xsource_unsorted(xsignature, states_p):
    """Restates the ``sorted_input=False`` branch of ``get_xsource`` (sqd.py:515-516, 542-545):
    uniquify with indices, the sorted-input algorithm, then
    ``arange(N).at[sort_indices].set(sort_indices[xsource])`` with -1 for missing sources.
    Unique rows without fill rows only (with repeats the reference scatters several values to
    one position, which JAX leaves unspecified)."""
    size = states_p.shape[0]
    srt, sort_indices = uniquify_states(states_p, size, return_indices=True)
    assert (sort_indices >= 0).all(), 'unique rows without fill rows only'
    xs = get_xsource(xsignature, srt).astype(np.int64)
    vals = np.where((xs >= 0) & (xs < size), sort_indices[np.clip(xs, 0, size - 1)], -1)
    out = np.arange(size, dtype=np.int64)
    out[sort_indices] = vals
    return out.astype(np.int32)


def get_xsource_dict(xsignature, states_p):
    """Independent dictionary lookup of S^X in S (cross-check of ``get_xsource`` on real rows)."""
    table = {row.tobytes(): i for i, row in enumerate(states_p) if row[0] != 255}
    mapped = np.bitwise_xor(states_p, xsignature)
    return np.array([table.get(row.tobytes(), -1) if states_p[i, 0] != 255 else -2
                     for i, row in enumerate(mapped)], dtype=np.int64)


def get_diagonal(zsignatures, coeffs, states):
    """Restates ``get_diagonal`` (sqd.py:603-628), including the stop at the first zero
    coefficient (:611-613)."""
    diagonal = np.zeros(states.shape[0], dtype=coeffs.dtype)
    for iterm in range(coeffs.shape[0]):
        if coeffs[iterm] == 0.:
            break
        bits = np.bitwise_count(states & zsignatures[iterm]).astype(np.int64)
        signed = np.sum(bits, axis=1) & 1
        signs = 1. - 2. * signed
        diagonal = diagonal + coeffs[iterm] * signs
    return diagonal


def apply_xgrp(xsource, diagonal, vec):
    """sqd.py:631-640: vec[xsource] * diagonal with 0 for out-of-range (incl. negative) indices."""
    valid = (xsource >= 0) & (xsource < vec.shape[0])
    xvec = np.zeros(xsource.shape[0], dtype=vec.dtype)
    xvec[valid] = vec[xsource[valid]]
    return xvec * diagonal


def apply_h_x_cached(vec, xsources, zsignatures, coeffs, states):
    """Restates ``apply_h_x_cached`` (sqd.py:694-709) on one device (offset 0, out zeros)."""
    out = np.zeros_like(vec, dtype=np.result_type(vec.dtype, coeffs.dtype))
    for xsource, zsigs, cs in zip(xsources, zsignatures, coeffs):
        out = out + apply_xgrp(xsource, get_diagonal(zsigs, cs, states), vec)
    return out


def apply_h(vec, xsignatures, zsignatures, coeffs, states):
    """Restates ``apply_h`` (sqd.py:643-658): uncached sources."""
    out = np.zeros_like(vec, dtype=np.result_type(vec.dtype, coeffs.dtype))
    for xsig, zsigs, cs in zip(xsignatures, zsignatures, coeffs):
        out = out + apply_xgrp(get_xsource(xsig, states), get_diagonal(zsigs, cs, states), vec)
    return out


def vinit_index(hamiltonian, states_u):
    """sqd.py:406-426: argmin of the group-0 diagonal over real rows if group 0 is X=0, else 0."""
    if np.all(hamiltonian.x[0] == 0):
        diagonal = get_diagonal(hamiltonian.z[0], hamiltonian.c[0], states_u).real
        diagonal = np.where(states_u[:, 0] == 255, np.inf, diagonal)
        return int(np.argmin(diagonal))
    return 0


def run_sqd(hamiltonian, states_p, states_size, options=None, xinit=None):
    """Restates ``run_sqd`` (sqd.py:317-442) with cache_strategy (1, 0) on one device.

    ``xinit`` (an extension used by tests) replaces the one-hot start vector.
    """
    if options is None:
        options = SQDOptions()
    states_u = uniquify_states(states_p, states_size)
    xsources = np.stack([get_xsource(x, states_u) for x in hamiltonian.x])

    def matvec(vec):
        return apply_h_x_cached(vec, xsources, hamiltonian.z, hamiltonian.c, states_u)

    vinit = vinit_index(hamiltonian, states_u) if xinit is None else xinit
    eigval, eigvec, niter = ground_locg(matvec, vinit, maxiter=options.locg_maxiter,
                                        tol=options.locg_tol,
                                        vspace=(states_size, hamiltonian.c.dtype))
    subspace_dim = int(np.searchsorted(states_u[:, 0] >> 7, 1))
    return eigval, eigvec, states_u, subspace_dim, niter


def sqd(hamiltonian, states, states_size=None, options=None, xinit=None):
    """Restates ``sqd`` (sqd.py:199-266)."""
    if isinstance(options, dict):
        options = SQDOptions(**options)
    if options is None:
        options = SQDOptions()
    if states_size is None:
        states_size = states.shape[0]
    if states_size < states.shape[0]:
        raise ValueError('states_size smaller than the states array length')
    if not isinstance(hamiltonian, PauliSumXZ):
        hamiltonian = from_paulisum(hamiltonian, force_real=True, add_padding=True)
    states_p = pack_states(states)
    eigval, eigvec, states_u, subspace_dim, niter = run_sqd(hamiltonian, states_p, states_size,
                                                            options, xinit=xinit)
    eigval = float(eigval)
    if options.return_eigvec:
        basis = np.unpackbits(states_u[:subspace_dim], axis=-1)[:, 1:1 + states.shape[1]]
        return eigval, np.array(eigvec[:subspace_dim]), basis
    return eigval


def hproj(hamiltonian, states, unique_states=False):
    """``hproj`` (sqd.py:269-314) with the padding mismatch fixed: the states are packed WITH the
    pad bit so that their byte width matches the padded Hamiltonian (sqd.py:295 vs :298).
    Returns (rows, cols, data) of the projected matrix in COO form, row-major sorted."""
    if not isinstance(hamiltonian, PauliSumXZ):
        hamiltonian = from_paulisum(hamiltonian, add_padding=True)
    if not unique_states:
        states = np.unique(states, axis=0)
    states_p = pack_states(states)
    rows_all, cols_all, data_all = [], [], []
    for x, z, c in zip(*hamiltonian.arrays):
        cols = get_xsource(x, states_p)
        diag = get_diagonal(z, c, states_p)
        valid = cols != -1
        rows_all.append(np.nonzero(valid)[0])
        cols_all.append(cols[valid])
        data_all.append(diag[valid])
    rows = np.concatenate(rows_all)
    cols = np.concatenate(cols_all)
    data = np.concatenate(data_all)
    order = np.lexsort((cols, rows))
    return rows[order], cols[order], data[order]


# ---------------------------------------------------------------------------------------------
# uint64 helpers (the representation the CUDA path uses): state value = sum_q s_q 2^q.
# ---------------------------------------------------------------------------------------------

def states_to_u64(states):
    """Binary [N, n] array in Qiskit order (last column = qubit 0) -> uint64 values."""
    states = np.asarray(states).astype(np.uint64)
    n = states.shape[1]
    weights = (np.uint64(1) << np.arange(n - 1, -1, -1, dtype=np.uint64))
    return (states * weights).sum(axis=1, dtype=np.uint64)


def u64_to_states(values, n):
    values = np.asarray(values, dtype=np.uint64)
    shifts = np.arange(n - 1, -1, -1, dtype=np.uint64)
    return ((values[:, None] >> shifts[None, :]) & np.uint64(1)).astype(np.uint8)


def packed_to_u64(packed, num_qubits):
    """Padded big-endian byte rows (pad bit first) -> uint64 values of the n qubit bits."""
    bits = np.unpackbits(packed, axis=-1)[..., 1:1 + num_qubits]
    return states_to_u64(bits.reshape(-1, num_qubits)).reshape(packed.shape[:-1])
