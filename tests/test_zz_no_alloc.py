"""sqd_vinit_noalloc, the allocation-free start-index search, checked against sqd_vinit, the
oracle's start index, and the library's memory pool.

Callers whose device memory is fully reserved by their own allocator cannot let the library
allocate; this entry point keeps its partial minima in a fixed __device__ array instead.  The
file is collected last so that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import _lib, workloads as W
from oracle import symplectic as OS, sqd as OQ

pytestmark = pytest.mark.gpu


def _vinit(name, op):
    idx = ctypes.c_int64(-1)
    _lib.check(getattr(_lib.load(), name)(op.handle, ctypes.byref(idx), _lib.stream_ptr()))
    return idx.value


def _operator(wl, cache=(1, 0), states_size=None):
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, wl.num_qubits, force_real=True,
                                padded=True)
    space = rq.Subspace.from_u64(wl.states, wl.num_qubits, states_size)
    return rq.SQDOperator(ham, space, cache_strategy=cache)


def test_noalloc_vinit_equals_vinit_on_two_calls_in_a_row():
    ops = [_operator(W.c1(0)), _operator(W.c2_small(0, 96, 80)),
           _operator(W.c1(3), cache=(0, 0), states_size=2100)]
    for op in ops:
        ref = _vinit('sqd_vinit', op)
        first = _vinit('sqd_vinit_noalloc', op)
        second = _vinit('sqd_vinit_noalloc', op)
        assert first == ref and second == ref
    # interleaved operators: the shared array keeps the previous call's contents
    for op in ops[::-1]:
        assert _vinit('sqd_vinit_noalloc', op) == _vinit('sqd_vinit', op)


def test_noalloc_vinit_without_diagonal_group_is_zero():
    rng = np.random.default_rng(0)
    x = np.array([3, 5, 6], dtype=np.uint64)
    z = np.array([0, 1, 4], dtype=np.uint64)
    ham = rq.PauliSumXZ.from_xz(x, z, rng.standard_normal(3), 4, force_real=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(np.arange(16, dtype=np.uint64), 4))
    assert _vinit('sqd_vinit_noalloc', op) == _vinit('sqd_vinit', op) == 0


def test_noalloc_vinit_rejects_subspaces_above_its_limit():
    n = (1 << 26) + 1                       # one state above the 67,108,864-row limit
    ham = rq.PauliSumXZ.from_xz(np.array([0], dtype=np.uint64), np.array([1], dtype=np.uint64),
                                np.array([1.0]), 27)
    space = rq.Subspace.from_u64(torch.arange(n, dtype=torch.int64, device='cuda'), 27)
    op = rq.SQDOperator(ham, space, cache_strategy=(0, 0))
    with pytest.raises(ValueError, match='67108864'):
        _vinit('sqd_vinit_noalloc', op)
    del op, space
    torch.cuda.empty_cache()


def test_noalloc_vinit_null_operator_is_an_error():
    idx = ctypes.c_int64()
    st = _lib.load().sqd_vinit_noalloc(None, ctypes.byref(idx), None)
    assert st == _lib.SQD_ERR_INVALID


def test_noalloc_vinit_matches_the_oracle_start_index():
    """vinit of run_sqd (sqd.py:406-426) as the oracle restates it."""
    for wl in (W.c1(0), W.c2_small(0, 96, 80)):
        op = _operator(wl)
        ham = OS.from_paulisum((wl.labels, list(wl.coeffs)), force_real=True, add_padding=True)
        su = OQ.pack_states(OQ.u64_to_states(wl.states, wl.num_qubits))
        assert _vinit('sqd_vinit_noalloc', op) == OQ.vinit_index(ham, su)


def test_noalloc_vinit_ties_keep_the_first_row():
    """Group 0 is a single Z on qubit 0: every odd state attains the minimum, and the first of
    them (in sorted order) is the start index, as jnp.argmin returns the first minimum."""
    states = np.array([2, 6, 7, 9, 12, 13, 15], dtype=np.uint64)
    ham = rq.PauliSumXZ.from_xz(np.array([0, 3], dtype=np.uint64),
                                np.array([1, 0], dtype=np.uint64), np.array([1.0, 0.25]), 4,
                                force_real=True)
    op = rq.SQDOperator(ham, rq.Subspace.from_u64(states, 4))
    assert _vinit('sqd_vinit_noalloc', op) == _vinit('sqd_vinit', op) == 2


def test_noalloc_vinit_allocates_nothing():
    """Warm calls leave the library pool's reserved bytes, live bytes and high-water mark, and
    torch's caching allocator, exactly as they were; the allocating sqd_vinit does move the
    high-water mark, so the check can see an allocation."""
    op = _operator(W.c2_small(0, 96, 80))
    _vinit('sqd_vinit_noalloc', op)               # the first call on the device: set-up
    torch.cuda.synchronize()
    torch_before = (torch.cuda.memory_allocated(), torch.cuda.memory_reserved())
    reserved0, used0, high0 = _lib.memory_stats(reset_high=True)
    assert high0 == used0
    for _ in range(3):
        _vinit('sqd_vinit_noalloc', op)
    torch.cuda.synchronize()
    assert _lib.memory_stats() == (reserved0, used0, used0)
    assert (torch.cuda.memory_allocated(), torch.cuda.memory_reserved()) == torch_before
    _lib.memory_stats(reset_high=True)
    _vinit('sqd_vinit', op)
    torch.cuda.synchronize()
    assert _lib.memory_stats()[2] > used0
