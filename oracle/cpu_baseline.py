"""Timed CPU baseline: the reference's default matvec algorithm on the host cores (test and
benchmark infrastructure only).

Restates apply_h_x_cached (sqd.py:694-709) with get_diagonal (sqd.py:603-628): for every X
group, the composed diagonal over the rows (one popcount pass per term, stopping at the first
zero coefficient) times the gathered source amplitudes, accumulated group by group.  Sources
are cached as in the reference's default cache_strategy (1, 0) (precomputed, not timed).
States are uint64 words instead of the reference's padded bytes (same bits, same arithmetic).

The rows are a bounded sample of the workload and the groups are split over a process pool
(spawn) so that every host core works; throughput is rows x terms / second.
"""
import multiprocessing as mp
import os
import time

import numpy as np

_W = {}


def group_terms(x, z, coeffs):
    """Group raw terms like PauliSumXZ.from_paulisum (symplectic.py:97-111): merge equal (x,z),
    groups ascending in x, terms ascending in z, phase (-i)^{|x&z|}."""
    x = np.asarray(x, dtype=np.uint64)
    z = np.asarray(z, dtype=np.uint64)
    coeffs = np.asarray(coeffs, dtype=np.complex128)
    keep = coeffs != 0
    x, z, coeffs = x[keep], z[keep], coeffs[keep]
    order = np.lexsort((z, x))
    x, z, coeffs = x[order], z[order], coeffs[order]
    new = np.concatenate([[True], (x[1:] != x[:-1]) | (z[1:] != z[:-1])])
    seg = np.cumsum(new) - 1
    c = np.zeros(int(seg[-1]) + 1, dtype=np.complex128)
    np.add.at(c, seg, coeffs)
    x, z = x[new], z[new]
    ph = np.bitwise_count(x & z).astype(np.int64) & 3
    c = c * np.array([1., -1j, -1., 1j])[ph]
    gstart = np.flatnonzero(np.concatenate([[True], x[1:] != x[:-1]]))
    gstart = np.append(gstart, x.shape[0])
    if np.all(c.imag == 0):
        c = c.real
    return x[gstart[:-1]], gstart, z, c


def _init(states_all, rows, gx, gstart, z, c, lo, hi):
    s = states_all[rows]
    srcs = []
    for j in range(lo, hi):
        t = s ^ gx[j]
        pos = np.searchsorted(states_all, t)
        pos = np.minimum(pos, states_all.shape[0] - 1)
        srcs.append(np.where(states_all[pos] == t, pos, -1))
    _W.update(s=s, gx=gx, gstart=gstart, z=z, c=c, lo=lo, hi=hi, srcs=srcs)


def _partial(v):
    s, gstart, z, c = _W['s'], _W['gstart'], _W['z'], _W['c']
    out = np.zeros(s.shape[0], dtype=np.result_type(v.dtype, c.dtype))
    for k, j in enumerate(range(_W['lo'], _W['hi'])):
        diag = np.zeros(s.shape[0], dtype=c.dtype)
        for t in range(gstart[j], gstart[j + 1]):
            if c[t] == 0:
                break
            diag = diag + c[t] * (1. - 2. * (np.bitwise_count(s & z[t]) & 1))
        src = _W['srcs'][k]
        xv = np.where(src >= 0, v[np.maximum(src, 0)], 0)
        out = out + xv * diag
    return out


class CpuMatvecSample:
    """The reference matvec restricted to ``rows`` (a sample), over ``nproc`` processes."""

    def __init__(self, x, z, coeffs, states, rows, nproc=None):
        self.gx, self.gstart, self.z, self.c = group_terms(x, z, coeffs)
        self.states = np.asarray(states, dtype=np.uint64)
        self.rows = np.asarray(rows)
        self.nproc = nproc or os.cpu_count() or 1
        self.num_terms = self.z.shape[0]
        J = self.gx.shape[0]
        # split groups so every worker gets a similar number of terms
        cum = self.gstart[1:]
        cuts = [0] + [int(np.searchsorted(cum, cum[-1] * k / self.nproc)) + 1
                      for k in range(1, self.nproc)] + [J]
        cuts = sorted(set(min(max(a, 0), J) for a in cuts))
        ctx = mp.get_context('spawn')
        self.pools = []
        for lo, hi in zip(cuts[:-1], cuts[1:]):
            if hi <= lo:
                continue
            pool = ctx.Pool(1, initializer=_init,
                            initargs=(self.states, self.rows, self.gx, self.gstart, self.z,
                                      self.c, lo, hi))
            self.pools.append(pool)

    def matvec(self, v):
        res = [p.apply_async(_partial, (v,)) for p in self.pools]
        out = res[0].get()
        for r in res[1:]:
            out = out + r.get()
        return out

    def time(self, v, reps=1):
        self.matvec(v)   # warm-up
        t0 = time.perf_counter()
        for _ in range(reps):
            self.matvec(v)
        return (time.perf_counter() - t0) / reps

    def close(self):
        for p in self.pools:
            p.terminate()
            p.join()


def projected_csr(x, z, coeffs, states):
    """The projected Hamiltonian <i|H|j> on sorted unique uint64 ``states`` as a SciPy CSR
    matrix (what ``hproj`` returns, sqd.py:269-314, with the states padded consistently): per X
    group, the sources by a sorted search (get_xsource's result for sorted unique rows) and the
    composed diagonal of get_diagonal (sqd.py:603-628) at the rows whose source exists."""
    import scipy.sparse as sps
    gx, gstart, zt, c = group_terms(x, z, coeffs)
    s = np.asarray(states, dtype=np.uint64)
    n = s.shape[0]
    rows, cols, data = [], [], []
    for j in range(gx.shape[0]):
        t = s ^ gx[j]
        pos = np.minimum(np.searchsorted(s, t), n - 1)
        ok = s[pos] == t
        if not ok.any():
            continue
        r = np.nonzero(ok)[0]
        diag = np.zeros(r.shape[0], dtype=c.dtype)
        for k in range(gstart[j], gstart[j + 1]):
            if c[k] == 0:
                break
            diag = diag + c[k] * (1. - 2. * (np.bitwise_count(s[r] & zt[k]) & 1))
        rows.append(r)
        cols.append(pos[r])
        data.append(diag)
    return sps.csr_matrix((np.concatenate(data), (np.concatenate(rows), np.concatenate(cols))),
                          shape=(n, n))
