"""Seeded synthetic SQD workloads: Pauli sums, Jordan-Wigner molecular Hamiltonians, subspaces.

Five standard workloads are defined (``c1`` ... ``c5``):

* ``c1``: 16-qubit random Pauli sum (300 draws, weight 1..4, N(0,1) coefficients), 2000 distinct
  weight-8 strings.
* ``c2``: Jordan-Wigner molecular Hamiltonian, 16 spatial orbitals (32 qubits, alpha = qubits
  0-15, beta = 16-31), 512 x 512 alpha/beta product subspace of 4-electron strings
  (D = 262,144).
* ``c3``: same construction with 24 orbitals (48 qubits), 4096 x 4096 strings of 6 electrons
  (D = 16,777,216).
* ``c4``: 96 c2-style instances with their own seeds, a_i x b_i strings, a_i, b_i log-uniform
  integers in [64, 1820].
* ``c5``: 40-qubit random Pauli sum (20,000 draws, N(0,1)/sqrt(M)), 1,048,576 distinct weight-20
  strings.

All random draws go through ``numpy.random.default_rng(seed)``.  The Pauli data is returned as
uint64 X/Z masks (bit q = qubit q) plus real coefficients; ``labels_from_xz`` produces the string
labels (character 0 = qubit n-1) for the tuple form of the public API.
"""
from dataclasses import dataclass, field
from itertools import combinations
import math
import numpy as np

U64 = np.uint64


# ---------------------------------------------------------------------------------------------
# Pauli label <-> mask conversion
# ---------------------------------------------------------------------------------------------

def labels_from_xz(x, z, n):
    """uint64 masks -> list of Pauli labels (character 0 = qubit n-1)."""
    x = np.asarray(x, dtype=U64)
    z = np.asarray(z, dtype=U64)
    shifts = np.arange(n - 1, -1, -1, dtype=U64)
    xb = ((x[:, None] >> shifts[None, :]) & U64(1)).astype(np.uint8)
    zb = ((z[:, None] >> shifts[None, :]) & U64(1)).astype(np.uint8)
    table = np.frombuffer(b'IZXY', dtype=np.uint8)
    chars = table[xb * 2 + zb]
    return [row.tobytes().decode() for row in chars]


def xz_from_labels(labels):
    """Pauli labels -> (x, z) uint64 masks and the number of qubits (n <= 64)."""
    if len(labels) == 0:
        raise ValueError('empty Pauli list')
    n = len(labels[0])
    raw = np.frombuffer(''.join(labels).upper().encode(), dtype=np.uint8).reshape(len(labels), n)
    xb = (raw == ord('X')) | (raw == ord('Y'))
    zb = (raw == ord('Y')) | (raw == ord('Z'))
    weights = U64(1) << np.arange(n - 1, -1, -1, dtype=U64)
    x = (xb.astype(U64) * weights).sum(axis=1, dtype=U64)
    z = (zb.astype(U64) * weights).sum(axis=1, dtype=U64)
    return x, z, n


# ---------------------------------------------------------------------------------------------
# Random Pauli sums
# ---------------------------------------------------------------------------------------------

def random_pauli_sum(n, m, rng, scale=1.0, wmin=1, wmax=4):
    """``m`` draws: weight uniform in wmin..wmax, support without replacement, Pauli uniform in
    {X, Y, Z}, coefficient N(0, 1) * scale.  Duplicates are NOT merged here (the Pauli-sum
    preprocessing merges them)."""
    x = np.zeros(m, dtype=U64)
    z = np.zeros(m, dtype=U64)
    weights = rng.integers(wmin, min(wmax, n) + 1, size=m)
    for t in range(m):
        support = rng.choice(n, size=weights[t], replace=False)
        kinds = rng.integers(0, 3, size=weights[t])   # 0 = X, 1 = Y, 2 = Z
        for q, k in zip(support, kinds):
            bit = U64(1) << U64(q)
            if k in (0, 1):
                x[t] |= bit
            if k in (1, 2):
                z[t] |= bit
    coeffs = rng.standard_normal(m) * scale
    return x, z, coeffs


def weight_subspace(n, k, d, rng):
    """``d`` distinct n-bit strings of Hamming weight ``k``, drawn uniformly, sorted (uint64)."""
    total = math.comb(n, k)
    if d > total:
        raise ValueError('subspace larger than the weight sector')
    if total <= 1 << 22:
        allv = np.array([sum(1 << q for q in c) for c in combinations(range(n), k)], dtype=U64)
        return np.sort(rng.choice(allv, size=d, replace=False))
    chosen = np.zeros(0, dtype=U64)
    while chosen.shape[0] < d:
        need = int((d - chosen.shape[0]) * 1.05) + 16
        keys = rng.random((need, n)).argsort(axis=1)[:, :k]
        vals = (U64(1) << keys.astype(U64)).sum(axis=1, dtype=U64)
        chosen = np.unique(np.concatenate([chosen, vals]))
    # unique() sorts; drop a uniformly random surplus
    if chosen.shape[0] > d:
        chosen = np.sort(rng.choice(chosen, size=d, replace=False))
    return chosen


def spin_strings(norb, nelec):
    """All ``norb``-bit strings with ``nelec`` ones, ascending."""
    return np.array(sorted(sum(1 << q for q in c) for c in combinations(range(norb), nelec)),
                    dtype=U64)


def product_subspace(norb, nelec, na, nb, rng):
    """Alpha (qubits 0..norb-1) x beta (qubits norb..2 norb-1) product of ``na`` x ``nb``
    strings sampled uniformly without replacement from the ``nelec``-electron strings."""
    total = math.comb(norb, nelec)
    if total <= 1 << 22:
        pool = spin_strings(norb, nelec)
        alpha = np.sort(rng.choice(pool, size=na, replace=False))
        beta = np.sort(rng.choice(pool, size=nb, replace=False))
    else:
        alpha = weight_subspace(norb, nelec, na, rng)
        beta = weight_subspace(norb, nelec, nb, rng)
    states = (beta[:, None] << U64(norb)) | alpha[None, :]
    return states.reshape(-1)          # beta-major: already ascending


# ---------------------------------------------------------------------------------------------
# Jordan-Wigner molecular Hamiltonians
# ---------------------------------------------------------------------------------------------

def random_integrals(norb, rng):
    """h1: symmetric, N(0,1)/16.  h2 (chemist's (ij|kl)): N(0, 0.1) with 8-fold symmetry."""
    a = rng.standard_normal((norb, norb)) / 16.
    h1 = np.triu(a) + np.triu(a, 1).T
    g = rng.normal(0., 0.1, size=(norb,) * 4)
    i, j, k, l = np.meshgrid(*(np.arange(norb),) * 4, indexing='ij')
    i0, j0 = np.minimum(i, j), np.maximum(i, j)
    k0, l0 = np.minimum(k, l), np.maximum(k, l)
    first = (i0 < k0) | ((i0 == k0) & (j0 <= l0))
    p0 = np.where(first, i0, k0)
    p1 = np.where(first, j0, l0)
    p2 = np.where(first, k0, i0)
    p3 = np.where(first, l0, j0)
    h2 = g[p0, p1, p2, p3]
    return h1, h2


def _ladder_products(ops, coef, n_qubits):
    """Expand sum_t coef[t] * prod_k ladder(ops[k][t]) into X^x Z^z monomials.

    ``ops`` is a list of (index array, dagger flag) in left-to-right product order.  A ladder
    operator on spin-orbital p is Z_{<p} X_p (I -/+ Z_p)/2 (annihilation/creation), i.e. the sum
    of the monomials X^{e_p} Z^{L_p} and X^{e_p} Z^{L_p + e_p} with weights 1/2 and -/+1/2.
    Multiplying monomials: (X^a Z^b)(X^c Z^d) = (-1)^{|b & c|} X^{a^c} Z^{b^d}.
    """
    nt = coef.shape[0]
    xs, zs, cs = [], [], []
    m = len(ops)
    for combo in range(1 << m):
        x = np.zeros(nt, dtype=U64)
        z = np.zeros(nt, dtype=U64)
        c = coef.astype(np.float64).copy()
        for k, (idx, dagger) in enumerate(ops):
            e = U64(1) << idx.astype(U64)
            low = e - U64(1)
            with_z = (combo >> k) & 1
            # sign from moving Z^z past X^e
            parity = (np.bitwise_count(z & e) & 1).astype(np.float64)
            c *= 1. - 2. * parity
            c *= 0.5 if (not with_z or dagger) else -0.5
            x ^= e
            z ^= (low | e) if with_z else low
        xs.append(x)
        zs.append(z)
        cs.append(c)
    x = np.concatenate(xs)
    z = np.concatenate(zs)
    c = np.concatenate(cs)
    # X^x Z^z = (-i)^{|x & z|} Q(x, z)
    ph = np.bitwise_count(x & z).astype(np.int64) & 3
    re = np.where(ph == 0, c, np.where(ph == 2, -c, 0.))
    im = np.where(ph == 1, -c, np.where(ph == 3, c, 0.))
    return x, z, re, im


def _merge(x, z, re, im):
    order = np.lexsort((z, x))
    x, z, re, im = x[order], z[order], re[order], im[order]
    start = np.concatenate([[True], (x[1:] != x[:-1]) | (z[1:] != z[:-1])])
    seg = np.cumsum(start) - 1
    nseg = int(seg[-1]) + 1
    re_s = np.bincount(seg, weights=re, minlength=nseg)
    im_s = np.bincount(seg, weights=im, minlength=nseg)
    return x[start], z[start], re_s, im_s


def jw_hamiltonian(h1, h2, cutoff=1e-12):
    """Jordan-Wigner qubit Hamiltonian of
    H = sum_{ij,s} h1_ij a+_{is} a_{js} + 1/2 sum_{ijkl,s,t} (ij|kl) a+_{is} a+_{kt} a_{lt} a_{js}
    with spin-orbital (i, s) on qubit i + s * norb.  Returns (x, z, coeff) with duplicates merged
    and |coeff| > cutoff, sorted by (x, z)."""
    norb = h1.shape[0]
    nq = 2 * norb
    parts = []
    # one-body
    i, j, s = np.meshgrid(np.arange(norb), np.arange(norb), np.arange(2), indexing='ij')
    i, j, s = i.ravel(), j.ravel(), s.ravel()
    c = h1[i, j]
    keep = c != 0.
    parts.append(_ladder_products([(i[keep] + norb * s[keep], True),
                                   (j[keep] + norb * s[keep], False)], c[keep], nq))
    # two-body
    i, j, k, l, s, t = np.meshgrid(*(np.arange(norb),) * 4, np.arange(2), np.arange(2),
                                   indexing='ij')
    i, j, k, l, s, t = (a.ravel() for a in (i, j, k, l, s, t))
    p = i + norb * s
    q = k + norb * t
    r = l + norb * t
    u = j + norb * s
    c = 0.5 * h2[i, j, k, l]
    keep = (p != q) & (r != u) & (c != 0.)
    chunk = 1 << 18
    idx = np.nonzero(keep)[0]
    for a0 in range(0, idx.shape[0], chunk):
        sel = idx[a0:a0 + chunk]
        part = _ladder_products([(p[sel], True), (q[sel], True), (r[sel], False),
                                 (u[sel], False)], c[sel], nq)
        parts.append(_merge(*part))
    x = np.concatenate([pt[0] for pt in parts])
    z = np.concatenate([pt[1] for pt in parts])
    re = np.concatenate([pt[2] for pt in parts])
    im = np.concatenate([pt[3] for pt in parts])
    x, z, re, im = _merge(x, z, re, im)
    if np.max(np.abs(im), initial=0.) > 1e-9:
        raise RuntimeError('JW Hamiltonian has imaginary coefficients')
    keep = np.abs(re) > cutoff
    return x[keep], z[keep], re[keep]


class JWStructure:
    """The Pauli terms of ``jw_hamiltonian`` for ``norb`` orbitals and the linear map from the
    independent integrals (h1 upper triangle, h2 canonical quadruples) to their coefficients,
    so that many instances with different integrals cost one sparse matvec each."""

    def __init__(self, norb):
        from scipy.sparse import coo_matrix
        self.norb = norb
        nq = 2 * norb
        idx1 = np.full((norb, norb), -1, dtype=np.int64)
        k = 0
        for i in range(norb):
            for j in range(i, norb):
                idx1[i, j] = idx1[j, i] = k
                k += 1
        self.n1 = k
        ii, jj, kk, ll = np.meshgrid(*(np.arange(norb),) * 4, indexing='ij')
        i0, j0 = np.minimum(ii, jj), np.maximum(ii, jj)
        k0, l0 = np.minimum(kk, ll), np.maximum(kk, ll)
        first = (i0 < k0) | ((i0 == k0) & (j0 <= l0))
        key = np.stack([np.where(first, i0, k0), np.where(first, j0, l0),
                        np.where(first, k0, i0), np.where(first, l0, j0)], axis=-1)
        flat = ((key[..., 0] * norb + key[..., 1]) * norb + key[..., 2]) * norb + key[..., 3]
        uniq, inv = np.unique(flat.ravel(), return_inverse=True)
        self.h2_keys = uniq
        self.idx2 = inv.reshape((norb,) * 4) + self.n1
        self.nparam = self.n1 + uniq.shape[0]
        xs, zs, res, ims, cols = [], [], [], [], []
        i, j, s = (a.ravel() for a in np.meshgrid(np.arange(norb), np.arange(norb),
                                                  np.arange(2), indexing='ij'))
        part = _ladder_products([(i + norb * s, True), (j + norb * s, False)],
                                np.ones(i.shape[0]), nq)
        reps = 4
        xs.append(part[0]); zs.append(part[1]); res.append(part[2]); ims.append(part[3])
        cols.append(np.tile(idx1[i, j], reps))
        i, j, k, l, s, t = (a.ravel() for a in np.meshgrid(*(np.arange(norb),) * 4, np.arange(2),
                                                           np.arange(2), indexing='ij'))
        p, q, r, u = i + norb * s, k + norb * t, l + norb * t, j + norb * s
        keep = (p != q) & (r != u)
        sel = np.nonzero(keep)[0]
        chunk = 1 << 17
        for a0 in range(0, sel.shape[0], chunk):
            sl = sel[a0:a0 + chunk]
            part = _ladder_products([(p[sl], True), (q[sl], True), (r[sl], False), (u[sl], False)],
                                    np.full(sl.shape[0], 0.5), nq)
            xs.append(part[0]); zs.append(part[1]); res.append(part[2]); ims.append(part[3])
            cols.append(np.tile(self.idx2[i[sl], j[sl], k[sl], l[sl]], 16))
        x = np.concatenate(xs)
        z = np.concatenate(zs)
        re = np.concatenate(res)
        im = np.concatenate(ims)
        col = np.concatenate(cols)
        order = np.lexsort((z, x))
        x, z = x[order], z[order]
        new = np.concatenate([[True], (x[1:] != x[:-1]) | (z[1:] != z[:-1])])
        row = np.cumsum(new) - 1
        nterm = int(row[-1]) + 1
        a_re = coo_matrix((re[order], (row, col[order])), shape=(nterm, self.nparam)).tocsr()
        a_im = coo_matrix((im[order], (row, col[order])), shape=(nterm, self.nparam)).tocsr()
        a_re.sum_duplicates()
        a_im.sum_duplicates()
        a_re.eliminate_zeros()
        if a_im.nnz:
            a_im.data[np.abs(a_im.data) < 1e-14] = 0.0
            a_im.eliminate_zeros()
        if a_im.nnz:
            raise RuntimeError('JW map has imaginary coefficients')
        a_re.data[np.abs(a_re.data) < 1e-15] = 0.0
        a_re.eliminate_zeros()
        live = np.diff(a_re.indptr) > 0
        self.x = x[new][live]
        self.z = z[new][live]
        self.map = a_re[live]

    def params(self, h1, h2):
        p = np.zeros(self.nparam)
        iu = np.triu_indices(self.norb)
        idx = np.full((self.norb, self.norb), -1)
        k = 0
        for i, j in zip(*iu):
            p[k] = h1[i, j]
            k += 1
        keys = self.h2_keys
        n = self.norb
        a, rem = np.divmod(keys, n ** 3)
        b, rem = np.divmod(rem, n ** 2)
        c, d = np.divmod(rem, n)
        p[self.n1:] = h2[a, b, c, d]
        return p

    def hamiltonian(self, h1, h2, cutoff=1e-12):
        """(x, z, coeff) of jw_hamiltonian(h1, h2) for symmetric h1 and 8-fold symmetric h2."""
        c = self.map @ self.params(h1, h2)
        keep = np.abs(c) > cutoff
        return self.x[keep], self.z[keep], c[keep]


# ---------------------------------------------------------------------------------------------
# Standard workloads
# ---------------------------------------------------------------------------------------------

@dataclass
class Workload:
    name: str
    num_qubits: int
    x: np.ndarray            # uint64 X masks of the raw terms
    z: np.ndarray            # uint64 Z masks
    coeffs: np.ndarray       # real coefficients
    states: np.ndarray       # sorted distinct uint64 states
    seed: int
    notes: dict = field(default_factory=dict)

    @property
    def labels(self):
        return labels_from_xz(self.x, self.z, self.num_qubits)

    def start_vector(self, dtype=np.complex128):
        rng = np.random.default_rng(self.seed + 7919)
        d = self.states.shape[0]
        v = rng.standard_normal(d)
        if np.dtype(dtype).kind == 'c':
            v = v + 1j * rng.standard_normal(d)
        v = v.astype(dtype)
        return v / np.linalg.norm(v)


def c1(seed=0):
    rng = np.random.default_rng(seed)
    x, z, c = random_pauli_sum(16, 300, rng)
    states = weight_subspace(16, 8, 2000, rng)
    return Workload('c1', 16, x, z, c, states, seed, {'tol': 1e-10})


def jw_workload(name, norb, nelec, na, nb, seed, structure=None):
    rng = np.random.default_rng(seed)
    h1, h2 = random_integrals(norb, rng)
    if structure is not None:
        x, z, c = structure.hamiltonian(h1, h2)
    else:
        x, z, c = jw_hamiltonian(h1, h2)
    states = product_subspace(norb, nelec, na, nb, rng)
    return Workload(name, 2 * norb, x, z, c, states, seed, {'norb': norb, 'nelec': nelec,
                                                             'na': na, 'nb': nb})


def c2(seed=0):
    return jw_workload('c2', 16, 4, 512, 512, seed)


def c2_small(seed=0, na=48, nb=40):
    """c2's Hamiltonian construction on a small product subspace (for oracle-sized checks)."""
    return jw_workload('c2_small', 16, 4, na, nb, seed)


def c3(seed=0):
    return jw_workload('c3', 24, 6, 4096, 4096, seed)


def c3_small(seed=0, na=1536, nb=1536):
    """c3's Hamiltonian construction on a 1536 x 1536 product subspace (D = 2,359,296): the
    same orbital count and pair classes at a size that full profiler captures allow."""
    return jw_workload('c3_small', 24, 6, na, nb, seed)


def c4_dims(seed=0, count=96):
    rng = np.random.default_rng(seed)
    lo, hi = math.log(64), math.log(1820)
    a = np.clip(np.rint(np.exp(rng.uniform(lo, hi, size=count))), 64, 1820).astype(int)
    b = np.clip(np.rint(np.exp(rng.uniform(lo, hi, size=count))), 64, 1820).astype(int)
    return a, b


def c4(seed=0, count=96, structure=None):
    """The batched workload: ``count`` 16-orbital JW instances with their own seeds (own
    integrals and subspaces).  The Pauli terms are shared, so the coefficients come from one
    ``JWStructure`` (built once, or passed in)."""
    a, b = c4_dims(seed, count)
    structure = structure or JWStructure(16)
    return [jw_workload(f'c4_{i}', 16, 4, int(a[i]), int(b[i]), seed * 1000 + 101 + i,
                        structure) for i in range(count)]


def c5(seed=0, m=20000, d=1 << 20):
    rng = np.random.default_rng(seed)
    x, z, c = random_pauli_sum(40, m, rng, scale=1. / math.sqrt(m))
    states = weight_subspace(40, 20, d, rng)
    return Workload('c5', 40, x, z, c, states, seed)


def notebook_case(seed, nq=12, nsample=100_000, nterm=100):
    """The recipe of the reference's tests/sqd.ipynb (seeded): random binary samples, random
    IXYZ strings, uniform(-1, 1) coefficients.  Returns (labels, coeffs, states[nsample, nq])."""
    rng = np.random.default_rng(seed)
    states = rng.choice(2, size=(nsample, nq)).astype(np.uint8)
    labels = [''.join('IXYZ'[ip] for ip in row) for row in rng.choice(4, size=(nterm, nq))]
    coeffs = rng.uniform(-1., 1., size=nterm)
    return labels, coeffs, states
