"""The row-sampled CPU matvec (``oracle.cpu_baseline``, the checker of the full-size GPU tests
and the timed CPU baseline) against the reference's own matvec outputs
(``tests/golden/reference_*.npz``, written by the unmodified reference)."""
import os

import numpy as np
import pytest

from oracle.cpu_baseline import CpuMatvecSample
from oracle import sqd as OQ
from rqutils_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
SUM_RTOL = 1e-13


def load(name):
    d = np.load(os.path.join(GOLDEN, name + '.npz'))
    return {k: d[k] for k in d.files}


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _sample_matvec(x, z, c, states, rows, v):
    cpu = CpuMatvecSample(x, z, c, states, rows, nproc=2)
    try:
        return cpu.matvec(v)
    finally:
        cpu.close()


def test_c1_all_rows_and_a_sample_match_the_reference_matvec():
    g = load('reference_c1')
    wl = W.c1(0)
    v = g['probes'][0]
    hv = _sample_matvec(wl.x, wl.z, wl.coeffs, wl.states, np.arange(2000), v)
    assert rel(hv, g['hv_10'][0]) < SUM_RTOL
    rows = np.sort(np.random.default_rng(3).choice(2000, size=300, replace=False))
    hv_rows = _sample_matvec(wl.x, wl.z, wl.coeffs, wl.states, rows, v)
    assert rel(hv_rows, g['hv_10'][0][rows]) < SUM_RTOL


@pytest.mark.parametrize('tag', ['evy12', 'jw8'])
def test_real_hamiltonians_match_the_reference_matvec(tag):
    g = load('reference_solves')
    lab = [s.decode() for s in g[f'{tag}_labels']]
    x, z, n = W.xz_from_labels(lab)
    states = np.unique(OQ.states_to_u64(g[f'{tag}_bits']))
    hv = _sample_matvec(x, z, g[f'{tag}_coeffs'], states, np.arange(states.shape[0]),
                        g[f'{tag}_probes'][0])
    assert rel(hv, g[f'{tag}_hv'][0]) < SUM_RTOL


@pytest.mark.parametrize('tag', ['evy12', 'jw8'])
def test_projected_csr_matches_the_reference_matvec(tag):
    from oracle.cpu_baseline import projected_csr
    g = load('reference_solves')
    lab = [s.decode() for s in g[f'{tag}_labels']]
    x, z, n = W.xz_from_labels(lab)
    states = np.unique(OQ.states_to_u64(g[f'{tag}_bits']))
    h = projected_csr(x, z, g[f'{tag}_coeffs'], states)
    assert rel(h @ g[f'{tag}_probes'][0], g[f'{tag}_hv'][0]) < SUM_RTOL
    assert abs(h - h.conj().T).max() == 0
