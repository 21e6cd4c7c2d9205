"""Autotuner for the matvec schedule and lookup method.

``tune_lanes`` times the cached matvec for every lanes-per-row choice (the number of warp
lanes that share one output row) with CUDA events and keeps the fastest for the precision of
the given vector dtype; ``tune_lookup`` compares the hash-table and binary-search lookups on the
connectivity build.  Results are cached per operator shape (rows, stored pairs, cache strategy,
dtype) for the process.
"""
import torch

_CACHE = {}


def _time(fn, reps):
    s = torch.cuda.current_stream()
    fn()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def tune_lanes(op, dtype, candidates=(2, 4, 8, 16, 32), reps=5, chunks=(0, 64, 256, 1024)):
    """Times every (lanes per row, chunk rows) schedule of the cached matvec for the precision
    of ``dtype`` and keeps the fastest."""
    if op.cache_strategy[0] != 1:
        return {'lanes_per_row': None, 'note': 'uncached matvec has a fixed schedule'}
    if op.value_complex and not dtype.is_complex:
        dtype = torch.complex128 if dtype == torch.float64 else torch.complex64
    precision = 0 if dtype in (torch.float64, torch.complex128) else 1
    key = (op.size, op.nnz, op.cache_strategy, dtype)
    if key in _CACHE:
        op.set_lanes(precision, _CACHE[key]['lanes_per_row'])
        op.set_chunk(precision, _CACHE[key]['chunk_rows'])
        return _CACHE[key]
    v = torch.randn(op.size, dtype=dtype, device=op.space.device)
    out = torch.empty_like(v)
    times = {}
    for ch in chunks:
        if ch and op.cache_strategy[1] != 2:
            continue                       # the chunked schedule is a CSR-kernel option
        op.set_chunk(precision, ch)
        for lpr in candidates:
            op.set_lanes(precision, lpr)
            times[(lpr, ch)] = _time(lambda: op.matvec(v, out), reps)
    best = min(times, key=times.get)
    op.set_lanes(precision, best[0])
    op.set_chunk(precision, best[1])
    res = {'lanes_per_row': best[0], 'chunk_rows': best[1],
           'ms': {f'{k[0]}/{k[1]}': round(t, 4) for k, t in times.items()}}
    _CACHE[key] = res
    return res


def tune_lookup(hamiltonian, space, cache_strategy=(1, 0)):
    """Builds the operator with each lookup method; returns (best, {method: seconds})."""
    import time
    from .sqd import SQDOperator
    times = {}
    for method in ('hash', 'bsearch'):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        SQDOperator(hamiltonian, space, cache_strategy, lookup=method)
        torch.cuda.synchronize()
        times[method] = time.perf_counter() - t0
    return min(times, key=times.get), times
