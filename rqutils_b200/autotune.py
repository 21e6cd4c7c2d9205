"""Autotuner for the matvec schedule and lookup method.

``tune_lanes`` times the cached matvec for every schedule — element layout (per-row pair
lists, or product slabs when the subspace is a product of high-half and low-half strings),
lanes per row (the number of warp lanes that share one output row) and rows per block chunk —
with CUDA events and keeps the fastest for the precision of the given vector dtype;
``tune_lookup`` compares the hash-table and binary-search lookups on the connectivity build.
Results are cached per operator shape (rows, stored pairs, cache strategy, dtype, layouts) for
the process.
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


def tune_lanes(op, dtype, candidates=(2, 4, 8, 16, 32), reps=5, chunks=(0, 64, 256, 1024),
               layouts=None):
    """Times every (layout, lanes per row, chunk rows) schedule of the cached matvec for the
    precision of ``dtype`` and keeps the fastest.  ``layouts`` defaults to 'csr' plus the
    product layouts when they apply (their lanes and chunks schedule the two-half pairs)."""
    if op.cache_strategy[0] != 1:
        return {'lanes_per_row': None, 'note': 'uncached matvec has a fixed schedule'}
    if op.value_complex and not dtype.is_complex:
        dtype = torch.complex128 if dtype == torch.float64 else torch.complex64
    precision = 0 if dtype in (torch.float64, torch.complex128) else 1
    if layouts is None:
        layouts = ('csr', 'product', 'product-csr') if op.has_product_layout else ('csr',)
    key = (op.size, op.nnz, op.cache_strategy, dtype, tuple(layouts))
    if key in _CACHE:
        best = _CACHE[key]
        op.set_layout(precision, best['layout'])
        op.set_lanes(precision, best['lanes_per_row'])
        op.set_chunk(precision, best['chunk_rows'])
        return best
    v = torch.randn(op.size, dtype=dtype, device=op.space.device)
    out = torch.empty_like(v)
    times = {}
    for layout in layouts:
        if op.cache_strategy[1] != 2 and layout != 'csr':
            continue
        op.set_layout(precision, layout)
        for ch in chunks:
            if ch and op.cache_strategy[1] != 2:
                continue                   # the chunked schedule is a CSR-kernel option
            op.set_chunk(precision, ch)
            for lpr in candidates:
                op.set_lanes(precision, lpr)
                times[(layout, lpr, ch)] = _time(lambda: op.matvec(v, out), reps)
    best = min(times, key=times.get)
    op.set_layout(precision, best[0])
    op.set_lanes(precision, best[1])
    op.set_chunk(precision, best[2])
    res = {'layout': best[0], 'lanes_per_row': best[1], 'chunk_rows': best[2],
           'ms': {f'{k[0]}/{k[1]}/{k[2]}': round(t, 4) for k, t in times.items()}}
    _CACHE[key] = res
    return res


def tune_lookup(hamiltonian, space, cache_strategy=(1, 0)):
    """Builds the operator with each lookup method ('product' only on product subspaces);
    returns (best, {method: seconds})."""
    import time
    from .sqd import SQDOperator
    from ._lib import SQDError
    times = {}
    for method in ('hash', 'bsearch', 'product'):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        try:
            SQDOperator(hamiltonian, space, cache_strategy, lookup=method)
        except SQDError:
            continue                         # 'product' on a subspace that is not a product
        torch.cuda.synchronize()
        times[method] = time.perf_counter() - t0
    return min(times, key=times.get), times
