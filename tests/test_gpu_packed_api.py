"""uniquify_states and get_xsource on the reference's packed byte rows (sqd.py:445-548), the
sorted and unsorted-input branches, against the CPU oracle: bit-exact."""
import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import workloads as W
from oracle import symplectic as OS, sqd as OQ

pytestmark = pytest.mark.gpu


def _rows(seed, n_rows=500, nq=11):
    rng = np.random.default_rng(seed)
    return OQ.pack_states(rng.integers(0, 2, size=(n_rows, nq)).astype(np.uint8)), rng


@pytest.mark.parametrize('nq', [7, 11, 30, 63])
def test_uniquify_states_packed_rows(nq):
    sp, rng = _rows(nq, 600, nq)
    sp = np.concatenate([sp, sp[rng.integers(0, 600, size=200)]])     # repeats
    sp = sp[rng.permutation(sp.shape[0])]
    n_u = np.unique(sp, axis=0).shape[0]
    for size in (n_u, n_u + 17, max(1, n_u - 9)):
        rows, idx = rq.uniquify_states(sp, size, return_indices=True)
        erows, eidx = OQ.uniquify_states(sp, size, return_indices=True)
        assert (rows.cpu().numpy() == erows).all()
        assert (idx.cpu().numpy() == eidx).all()
        assert (rq.uniquify_states(torch.as_tensor(sp), size).cpu().numpy() == erows).all()


def test_uniquify_states_with_fill_rows_in_the_input():
    sp, _ = _rows(3, 300, 9)
    sp = np.concatenate([sp[:100], np.full((3, sp.shape[1]), 255, np.uint8), sp[100:]])
    n_u = np.unique(sp, axis=0).shape[0]
    rows, idx = rq.uniquify_states(sp, n_u + 4, return_indices=True)
    erows, eidx = OQ.uniquify_states(sp, n_u + 4, return_indices=True)
    assert (rows.cpu().numpy() == erows).all() and (idx.cpu().numpy() == eidx).all()


@pytest.mark.parametrize('lookup', ['hash', 'bsearch'])
def test_get_xsource_packed_sorted_rows_with_fill(lookup):
    labels, coeffs, states = W.notebook_case(5, nq=9, nsample=300, nterm=30)
    ham = OS.from_paulisum((labels, list(coeffs)), force_real=True, add_padding=True)
    sp = OQ.uniquify_states(OQ.pack_states(states), 350)
    for x in ham.x:
        got = rq.get_xsource(x, sp, lookup=lookup).cpu().numpy()
        assert (got == OQ.get_xsource(x, sp)).all()
    # device tensors in, as a caller holding them on the GPU would pass them
    x = ham.x[1]
    got = rq.get_xsource(torch.as_tensor(x).cuda(), torch.as_tensor(sp).cuda(), lookup=lookup)
    assert (got.cpu().numpy() == OQ.get_xsource(x, sp)).all()


def test_get_xsource_packed_unsorted_rows():
    sp, rng = _rows(5, 800, 12)
    sp = np.unique(sp, axis=0)
    rows = sp[rng.permutation(sp.shape[0])]
    xs = OQ.pack_states(rng.integers(0, 2, size=(8, 12)).astype(np.uint8))
    xs = np.concatenate([xs, np.zeros((1, xs.shape[1]), np.uint8)])   # x = 0: identity
    for x in xs:
        got = rq.get_xsource(x, rows, sorted_input=False).cpu().numpy()
        assert (got == OQ.get_xsource_unsorted(x, rows)).all()
    # sorted rows: both branches agree
    x = xs[0]
    assert (rq.get_xsource(x, sp, sorted_input=False).cpu().numpy()
            == rq.get_xsource(x, sp).cpu().numpy()).all()


def test_get_xsource_packed_rejects_what_the_reference_leaves_undefined():
    sp, rng = _rows(6, 200, 8)
    uniq = np.unique(sp, axis=0)
    x = uniq[1] ^ uniq[0]
    with pytest.raises(ValueError):
        rq.get_xsource(x, uniq[::-1].copy())                        # not sorted
    with pytest.raises(ValueError):
        rq.get_xsource(x, sp, sorted_input=False)                    # repeated rows
    with pytest.raises(ValueError):
        rq.get_xsource(x, OQ.uniquify_states(uniq, uniq.shape[0] + 3), sorted_input=False)
    with pytest.raises(ValueError):
        rq.get_xsource(x[:1], uniq)                                  # byte count mismatch


@pytest.mark.parametrize('lookup', ['hash', 'bsearch'])
def test_subspace_lookup_of_arbitrary_keys(lookup):
    rng = np.random.default_rng(9)
    states = np.unique(rng.integers(0, 1 << 20, size=3000).astype(np.uint64))
    space = rq.Subspace.from_u64(states, 20)
    keys = np.concatenate([states[rng.permutation(states.shape[0])[:500]],
                           rng.integers(0, 1 << 20, size=500).astype(np.uint64),
                           np.array([1 << 20, (1 << 63) + 5, (1 << 64) - 1], dtype=np.uint64)])
    got = space.lookup(torch.as_tensor(keys.view(np.int64)), lookup).cpu().numpy()
    expect = np.searchsorted(states, keys)
    found = (expect < states.shape[0]) & (states[np.minimum(expect, states.shape[0] - 1)] == keys)
    assert (got == np.where(found, expect, -1)).all()
