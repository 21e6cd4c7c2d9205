"""Benchmark of the SQD hot path on B200.

Default workload (one GPU): the 48-qubit Jordan-Wigner molecular Hamiltonian (24 spatial
orbitals, h1 ~ N(0,1)/16, h2 ~ N(0,0.1) with 8-fold symmetry, seed 0, 485,281 merged terms) on
the 4096 x 4096 alpha/beta product subspace of 6-electron strings (D = 16,777,216), complex128
vectors: the mixed-precision single-instance configuration.  ``--workload c2`` selects the
32-qubit, 16-orbital construction on 512 x 512 4-electron strings (D = 262,144).

A step is one Pauli-sum matvec Hv over the whole subspace (the inner kernel of LOCG).  ``value``
is row.terms/s = (rows x merged terms) / step time, summed over ranks (replicas, weak scaling),
with inputs resident in HBM; ``e2e`` is the same metric through the public API with every
step's input vector copied from pinned host memory and its result copied back inside the
timed region (copies of neighbouring steps overlap the matvec on separate streams).
Beside it: the roofline of the matvec (its kernels together), the LOCG time-to-E0 (FP64 and
mixed precision),
and the CPU baseline (the reference's default matvec algorithm on the host cores, on a fixed
seeded row sample).  ``--impl reference`` times only that CPU path, on the same row sample, so
the two CPU figures measure the same work.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--workload c3|c2|c1|c5|c4] [--cache 1,0|1,2|0,0] [--no-locg]
                       [--precision fp64|fp32]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'matvec row.terms/s (SQD Pauli-sum matvec over the sampled subspace)'
UNIT = 'row.terms/s'


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default='c3', choices=['c1', 'c2', 'c3', 'c4', 'c5', 'c3_small'])
    ap.add_argument('--cache', default='1,2')
    ap.add_argument('--no-locg', action='store_true')
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--no-graph', action='store_true',
                    help='LOCG without CUDA graphs (so a profiler sees every pass kernel)')
    ap.add_argument('--cpu-rows', type=int, default=0,
                    help='CPU sample rows (0 = the workload\'s fixed sample)')
    ap.add_argument('--lanes', type=int, default=0, help='lanes per row (0 = autotune)')
    ap.add_argument('--chunk', type=int, default=0, help='rows per block chunk with --lanes')
    ap.add_argument('--layout', default='csr', choices=['csr', 'product', 'product-csr'],
                    help='element layout with --lanes (the autotuner picks it otherwise)')
    ap.add_argument('--precision', default='fp64', choices=['fp64', 'fp32'],
                    help='vectors of the timed matvec: complex128 (default) or complex64 with '
                         'FP32 elements and compensated sums (the bulk of the mixed solver)')
    return ap.parse_args()


def make_workload(name):
    from rqutils_b200 import workloads as W
    return {'c1': W.c1, 'c2': W.c2, 'c3': W.c3, 'c5': W.c5, 'c3_small': W.c3_small}[name](0)


def workload_config(wl, cache, world=1):
    """The workload a line measures (identical in both arms)."""
    cfg = {'workload': f'{wl.name}: {wl.num_qubits}-qubit '
                       + ('JW molecular Hamiltonian, alpha x beta product subspace'
                          if wl.name in ('c2', 'c3', 'c3_small') else 'random Pauli sum, weight subspace'),
           'num_qubits': wl.num_qubits, 'subspace_dim': int(wl.states.shape[0]),
           'raw_terms': int(wl.coeffs.shape[0]), 'seed': wl.seed,
           'cache_strategy': list(cache), 'vector_dtype': 'complex128',
           'l2': 'no flush: stored pairs read per step exceed the 126 MB L2'}
    cfg.update({k: v for k, v in wl.notes.items() if k in ('norb', 'nelec', 'na', 'nb')})
    cfg['parallelism'] = f'replicas x{world}'
    return cfg


def load_peaks():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d['hbm_gbs']), 'measured'
    return 6650.0, 'fallback'


# Sources of the matvec kernels (and the headers they include): the traffic of a committed
# profile summary is used only while these are unchanged.
MATVEC_SOURCES = ('accum.cuh', 'common.cuh', 'dispatch.cuh', 'internal.cuh', 'matvec.cu',
                  'product.cu', 'sweep.cuh')


def kernel_sources_digest():
    """SHA-256 over the matvec kernels' sources (name and bytes, sorted by name): identifies
    the kernels a profile summary was captured on."""
    import hashlib
    csrc = os.path.join(ROOT, 'rqutils_b200', 'csrc')
    h = hashlib.sha256()
    for name in sorted(MATVEC_SOURCES):
        h.update(name.encode())
        with open(os.path.join(csrc, name), 'rb') as f:
            h.update(f.read())
    return h.hexdigest()


def load_traffic(workload, cache, layout='csr', precision='fp64'):
    """DRAM traffic of one matvec (all its kernels) from the committed ncu summary of this
    workload, layout and precision (FP32 vectors: suffix _fp32).  Used only when the summary's
    ``kernel_sources_sha256`` equals the digest of the current sources; otherwise (kernels
    changed since the capture) the traffic is reported as unknown.  Returns (bytes, note)."""
    names = [''] if layout == 'csr' else [f'_{layout}', '_product', '_product-csr']
    suffix = '' if precision == 'fp64' else '_' + precision
    paths = [os.path.join(ROOT, 'profiles',
                          f'matvec_{workload}_cache{cache[0]}{cache[1]}{n}{suffix}.md')
             for n in names]
    paths = [p for p in paths if os.path.exists(p)]
    if not paths:
        return None, 'no ncu summary for this workload/layout'
    fields = {}
    with open(paths[0]) as f:
        for line in f:
            if ':' in line and line.split(':', 1)[0].strip() in (
                    'traffic_bytes_per_launch', 'kernel_sources_sha256'):
                k, v = line.split(':', 1)
                fields[k.strip()] = v.strip()
    rel = os.path.relpath(paths[0], ROOT)
    if fields.get('kernel_sources_sha256') != kernel_sources_digest():
        return None, f'{rel} was captured on other kernel sources'
    if 'traffic_bytes_per_launch' not in fields:
        return None, f'{rel} has no traffic line'
    return float(fields['traffic_bytes_per_launch']), f'ncu capture in {rel}'


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', f'--id={self.index}', f'--query-gpu={self.QUERY}',
                 '--format=csv,noheader,nounits', '-lms', '100'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in self.lines:
            parts = [p.strip() for p in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == 'active':
                    reasons.add(name)
        if not sm:
            return None
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': max(mx),
                'reasons': sorted(reasons), 'samples': len(sm)}


def init_dist(n_gpus):
    import torch
    import torch.distributed as dist
    if n_gpus <= 1 or 'RANK' not in os.environ:
        return 0, 1, None
    from datetime import timedelta
    local = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(local)
    dist.init_process_group('nccl', timeout=timedelta(seconds=120),
                            device_id=torch.device('cuda', local))
    return dist.get_rank(), dist.get_world_size(), dist


def max_over_ranks(val, dist, device='cuda'):
    """Slowest rank's time: every rank takes part in the same collective."""
    if dist is None:
        return val
    import torch
    t = torch.tensor([val], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(val, dist, device='cuda'):
    """Whole-job total of per-rank work units."""
    if dist is None:
        return val
    import torch
    t = torch.tensor([val], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def replica_throughput(units_per_step, steps, t_local, dist, device='cuda'):
    """value = units all ranks processed / max-over-ranks time (replicas, weak scaling)."""
    t_max = max_over_ranks(t_local, dist, device)
    return sum_over_ranks(units_per_step * steps, dist, device) / t_max, t_max


def barrier(dist):
    import torch
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()


# Rows of the CPU sample per workload: about 1-3 s of host work per step on 16 cores.  The
# cpu_baseline leg and the --impl reference arm time the same seeded sample.
CPU_SAMPLE_ROWS = {'c1': 2000, 'c2': 32768, 'c3': 2048, 'c3_small': 8192, 'c5': 65536}


def cpu_sample(wl, rows=0):
    n = wl.states.shape[0]
    rows = rows or CPU_SAMPLE_ROWS.get(wl.name, 16384)
    rows = min(rows, n)
    rng = np.random.default_rng(1)
    return np.sort(rng.choice(n, size=rows, replace=False))


def cpu_sample_desc(sample, n, m, extra=''):
    return (f'{sample.shape[0]} of {n} rows (seeded uniform sample, rng 1), all {m} merged '
            f'terms, one matvec per step{extra}; NumPy restatement of apply_h_x_cached + '
            'get_diagonal (sqd.py:603-709) over a spawn process pool on every host core')


def cpu_baseline(wl, rows=0):
    """The reference's default matvec on the host cores over the workload's fixed row sample
    (one warm-up step, one timed step)."""
    from oracle.cpu_baseline import CpuMatvecSample
    n = wl.states.shape[0]
    sample = cpu_sample(wl, rows)
    cpu = CpuMatvecSample(wl.x, wl.z, wl.coeffs, wl.states, sample)
    v = wl.start_vector(np.complex128)
    t1 = cpu.time(v, reps=1)
    m = cpu.num_terms
    cpu.close()
    return {'value': sample.shape[0] * m / t1, 'unit': UNIT, 'cores': cpu.nproc,
            'kind': 'port', 'sample': cpu_sample_desc(sample, n, m, f' ({t1:.2f} s)')}


def run_reference(args):
    """The reference arm: the oracle port of the reference's default matvec (the reference
    itself needs JAX, absent from this image) on every host core, on the same seeded row
    sample as the cpu_baseline leg.  Maps no library of this repository."""
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    if args.workload == 'c4':
        print(json.dumps({'impl': 'reference', 'unavailable':
                          'c4 is a batched-solver workload; the CPU port times matvecs only'}),
              flush=True)
        return
    wl = make_workload(args.workload)
    from oracle.cpu_baseline import CpuMatvecSample
    n = wl.states.shape[0]
    sample = cpu_sample(wl, args.cpu_rows)
    cpu = CpuMatvecSample(wl.x, wl.z, wl.coeffs, wl.states, sample)
    v = wl.start_vector(np.complex128)
    for _ in range(max(0, args.warmup)):
        cpu.matvec(v)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu.matvec(v)
    dt = (time.perf_counter() - t0) / max(1, args.steps)
    cpu.close()
    val = sample.shape[0] * cpu.num_terms / dt
    line = {'impl': 'reference', 'metric': METRIC, 'value': val, 'unit': UNIT,
            'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': dt * 1e3, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'complex128 (f64 arithmetic)', 'data': 'synthetic',
            'config': workload_config(wl, tuple(int(v) for v in args.cache.split(',')),
                                      args.gpus),
            'cpu_baseline': {'value': val, 'unit': UNIT, 'cores': cpu.nproc, 'kind': 'port',
                             'sample': cpu_sample_desc(sample, n, cpu.num_terms) +
                                       ' (the same Hv as every cache strategy; the reference\'s '
                                       'default (1, 0) algorithm)'},
            'e2e': {'value': val, 'unit': UNIT, 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    rank, world, dist = init_dist(args.gpus)
    if world == 1:
        torch.cuda.set_device(0)
    dev = torch.device('cuda', torch.cuda.current_device())
    import rqutils_b200 as rq

    cache = tuple(int(v) for v in args.cache.split(','))
    wl = make_workload(args.workload)
    ham = rq.PauliSumXZ.from_xz(wl.x, wl.z, wl.coeffs, wl.num_qubits, force_real=True,
                                padded=True)
    space = rq.Subspace.from_u64(wl.states, wl.num_qubits)
    torch.cuda.synchronize()
    from rqutils_b200 import _lib
    used0 = _lib.memory_stats()[1]
    t_setup0 = time.perf_counter()
    op = rq.SQDOperator(ham, space, cache_strategy=cache)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t_setup0
    used_op = _lib.memory_stats()[1] - used0
    if args.lanes:
        for prec in (0, 1):
            op.set_layout(prec, args.layout)
            op.set_chunk(prec, args.chunk)
        op.lanes_per_row = args.lanes
        tuned = {'layout': args.layout, 'lanes_per_row': args.lanes, 'chunk_rows': args.chunk,
                 'note': 'fixed by --layout/--lanes/--chunk'}
    else:
        tuned = op.autotune()
    torch.cuda.synchronize()
    used_tuned = _lib.memory_stats()[1] - used0
    n_rows = space.states_size
    m_terms = ham.num_terms
    j_groups = ham.num_groups
    nnz = op.nnz

    prec = 0 if args.precision == 'fp64' else 1
    v = torch.as_tensor(wl.start_vector(np.complex128 if prec == 0 else np.complex64), device=dev)
    out = torch.empty_like(v)
    stream = torch.cuda.current_stream()
    for _ in range(max(3, args.warmup)):
        op.matvec(v, out)
    sampler = ClockSampler(dev.index) if rank == 0 else None
    barrier(dist)
    if sampler:
        sampler.start()
        time.sleep(0.3)
    barrier(dist)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # NVTX range 'timed_matvec': a profiler can select exactly these launches
    # (ncu --nvtx --nvtx-include "timed_matvec]")
    torch.cuda.nvtx.range_push('timed_matvec')
    ev0.record(stream)
    for _ in range(args.steps):
        op.matvec(v, out)
    ev1.record(stream)
    torch.cuda.nvtx.range_pop()
    barrier(dist)
    t_local = ev0.elapsed_time(ev1) / 1e3
    units = n_rows * m_terms
    value, t_max = replica_throughput(units, args.steps, t_local, dist)
    # kernels per matvec: CSR layout 1; product layout: transpose, low-half slabs, transpose,
    # two-half CSR tails (when there are any), high-half slabs
    layout = op.get_layout(prec) if cache == (1, 2) else 'csr'
    per_step = 1
    if layout in ('product', 'product-csr'):
        per_step = 5 if op.product_info()['pairs_mixed'] > 0 else 4
    gpu_launches = args.steps * per_step

    # end to end: pinned host input -> device -> matvec -> pinned host output, every step.
    # Three streams and two buffer sets pipeline the steps: the copy of step i+1's input and
    # the copy-out of step i-1's result overlap step i's matvec (PCIe is full duplex).
    e2e_s = e2e_pipelined(op, v, args.steps)
    barrier(dist)
    e2e_value, _ = replica_throughput(units, args.steps, e2e_s, dist)
    clocks = sampler.stop() if sampler else None
    step_s = t_max / args.steps

    # roofline of the matvec kernel (algorithmic bytes per launch)
    w_v, w_c, W = v.element_size(), 16, 1
    bytes_alg = n_rows * (8 * W + 2 * w_v) + nnz * w_v + m_terms * (8 * W + w_c) + j_groups * 8 * W
    peak, peak_kind = load_peaks()
    achieved = bytes_alg / (t_local / args.steps) / 1e9
    traffic, traffic_note = load_traffic(args.workload, cache, layout, args.precision)
    dram_frac = None
    if traffic is not None:
        dram_frac = traffic / (t_local / args.steps) / 1e9 / peak
    props = torch.cuda.get_device_properties(dev)
    sm_mhz = clocks['sm_mhz'] if clocks and clocks.get('sm_mhz') else 1965.0
    issue = None
    if prec == 0:
        issue = issue_bound(n_rows, m_terms, nnz, op.value_complex,
                            props.multi_processor_count, sm_mhz, t_local / args.steps)

    extra = {}
    if not args.no_locg and rank == 0:
        extra['locg'] = locg_times(rq, op, wl, dev, use_graph=not args.no_graph)
        extra['locg']['bytes_per_iteration'] = locg_bytes(n_rows, m_terms, j_groups, nnz)
    if args.workload == 'c5' and rank == 0:
        extra['gradient'] = gradient_check(rq, op, wl)
    line = None
    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': step_s * 1e3,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': ('complex128 (f64 arithmetic)' if prec == 0 else
                      'complex64 (f32 products, compensated sums, f64 partials)'),
            'data': 'synthetic (seeded generator)',
            'config': workload_config(wl, cache, world),
            'schedule': {'merged_terms': m_terms, 'x_groups': j_groups, 'stored_pairs': nnz,
                         'lanes_per_row': {'fp64': op.get_lanes(0), 'fp32': op.get_lanes(1)},
                         'layout': {'fp64': layout,
                                    'fp32': op.get_layout(1) if cache == (1, 2) else 'csr'},
                         'kernels_per_matvec': per_step, 'precision': args.precision,
                         'autotune': tuned, 'setup_s': setup_s,
                         'device_memory_bytes': {
                             'operator': used_op, 'with_layouts': used_tuned,
                             'note': 'library pool bytes in use for this cache strategy: the '
                                     'operator as built, then with the matvec layouts the '
                                     'schedule selected (FP32 copies, product slabs)'}},
            'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak, 'traffic': traffic,
                         'traffic_source': traffic_note,
                         'dram_frac': dram_frac,
                         'peak_kind': peak_kind,
                         'bytes_alg_per_launch': bytes_alg,
                         'formula': 'N(8W+2w_v) + P_valid w_v + M(8W+w_c) + J 8W, W=1, '
                                    f'w_v={w_v}, w_c=16, P_valid = stored pairs',
                         'timed': f'one whole {args.precision.upper()} matvec (all its kernels) '
                                  'per launch'},
            'issue_bound': issue,
            'e2e': {'value': e2e_value, 'unit': UNIT,
                    'h2d_bytes_per_step': int(v.numel() * v.element_size()),
                    'd2h_bytes_per_step': int(v.numel() * v.element_size())},
            'gpu_launches': gpu_launches,
            'clocks': clocks,
        }
        line.update(extra)
    if rank == 0 and world == 1 and not args.no_cpu:
        line['cpu_baseline'] = cpu_baseline(wl, rows=args.cpu_rows)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def e2e_pipelined(op, v, steps):
    """Seconds for ``steps`` matvecs whose inputs come from pinned host memory and whose
    results go back to pinned host memory, pipelined over copy-in, compute and copy-out
    streams with two device buffer sets (warm-up of two steps first)."""
    import torch
    s_in, s_mv, s_out = (torch.cuda.Stream() for _ in range(3))
    v_host = v.cpu().pin_memory()
    o_host = [torch.empty_like(v_host).pin_memory() for _ in range(2)]
    v_dev = [torch.empty_like(v) for _ in range(2)]
    o_dev = [torch.empty_like(v) for _ in range(2)]
    ev = lambda: torch.cuda.Event()
    in_done = [ev(), ev()]
    mv_done = [ev(), ev()]
    out_done = [ev(), ev()]
    for e in mv_done + out_done:
        e.record(torch.cuda.current_stream())

    def step(i):
        b = i % 2
        with torch.cuda.stream(s_in):
            s_in.wait_event(mv_done[b])            # step i-2 no longer reads v_dev[b]
            v_dev[b].copy_(v_host, non_blocking=True)
            in_done[b].record(s_in)
        with torch.cuda.stream(s_mv):
            s_mv.wait_event(in_done[b])
            s_mv.wait_event(out_done[b])           # step i-2's result has left o_dev[b]
            op.matvec(v_dev[b], o_dev[b])
            mv_done[b].record(s_mv)
        with torch.cuda.stream(s_out):
            s_out.wait_event(mv_done[b])
            o_host[b].copy_(o_dev[b], non_blocking=True)
            out_done[b].record(s_out)

    for i in range(2):
        step(i)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(s_in)
    for i in range(steps):
        step(i)
    t1.record(s_out)
    t1.synchronize()
    ms = t0.elapsed_time(t1)
    torch.cuda.synchronize()
    return ms / 1e3


def gradient_check(rq, op, wl, n_coords=32, h=1e-5):
    """dE0/dc for every raw coefficient through the autograd backward (Hellmann-Feynman),
    against FP64 central finite differences on ``n_coords`` random coordinates."""
    import torch
    from rqutils_b200.autograd import ground_energy
    coeffs = torch.as_tensor(wl.coeffs, device='cuda').clone().requires_grad_(True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e = ground_energy(coeffs, op)
    e.backward()
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t0
    grad = coeffs.grad.detach().cpu().numpy()
    rng = np.random.default_rng(5)
    ks = rng.choice(len(wl.coeffs), size=n_coords, replace=False)
    errs = []
    t0 = time.perf_counter()
    for k in ks:
        cp = wl.coeffs.copy()
        cm = wl.coeffs.copy()
        cp[k] += h
        cm[k] -= h
        ep = ground_energy(torch.as_tensor(cp, device='cuda'), op).item()
        em = ground_energy(torch.as_tensor(cm, device='cuda'), op).item()
        fd = (ep - em) / (2 * h)
        errs.append(abs(fd - grad[k]) / max(abs(fd), 1e-12))
    t_fd = time.perf_counter() - t0
    ground_energy(torch.as_tensor(wl.coeffs, device='cuda'), op)   # restore
    return {'energy': e.item(), 'num_coeffs': int(len(wl.coeffs)),
            'time_energy_and_gradient_s': t_grad, 'fd_coords': int(n_coords), 'fd_step': h,
            'fd_time_s': t_fd, 'max_rel_err_vs_fd': float(max(errs)),
            'median_rel_err_vs_fd': float(np.median(errs))}


POPC_PER_SM_CLK = 16      # 32-bit population count results per SM per clock (sm_90/sm_100)
DFMA_PER_SM_CLK = 64      # FP64 fused multiply-adds per SM per clock (B200: 148 SMs, ~37 TF/s)


def issue_bound(n, m, p, value_complex, sms, sm_mhz, t_matvec_s):
    """Instruction-issue floors of one FP64 matvec, beside its memory roofline.

    The reference's matvec (apply_h_x_cached, sqd.py:694-709) recomputes every group's diagonal
    (get_diagonal, sqd.py:603-628) for every row and merged term: N x M population counts per
    matvec.  The timed kernels read cached elements instead: one FP64 complex-by-real (2 FMAs)
    or complex-by-complex (4 FMAs) product per stored pair.  Both are divided by the nominal
    per-SM throughputs at the sampled SM clock."""
    hz = sms * sm_mhz * 1e6
    popc = n * m
    fma = p * (4 if value_complex else 2)
    return {'reference_popcounts_per_matvec': popc,
            'reference_popcount_floor_ms': popc / (POPC_PER_SM_CLK * hz) * 1e3,
            'cached_fp64_fma_per_matvec': fma,
            'cached_fp64_fma_floor_ms': fma / (DFMA_PER_SM_CLK * hz) * 1e3,
            'timed_matvec_ms': t_matvec_s * 1e3,
            'sms': sms, 'sm_mhz': sm_mhz,
            'rates': f'nominal: {POPC_PER_SM_CLK} popc and {DFMA_PER_SM_CLK} FP64 FMA '
                     'per SM per clock'}


def locg_bytes(n, m, j, p):
    """Algorithmic bytes of one LOCG iteration: matvecs x the matvec formula (W = 1, w_c = 16)
    plus the vector reads and writes of the fused passes, counted from the iteration bodies:
    the FP64 reference iteration (ground_locg.py:324-383) makes 4 complex128 matvecs and 42
    vector reads/writes; an FP32 sweep of the mixed solver 1 complex64 matvec and 33 as a graph
    of passes, 20 in the persistent launch (operators of at most 4 Mi rows and 64 Mi stored
    pairs: C1, C5)."""
    def mv(w_v):
        return n * (8 + 2 * w_v) + p * w_v + m * (8 + 16) + j * 8
    persistent = n <= (4 << 20) and p <= (64 << 20)
    return {'fp64': 4 * mv(16) + 42 * n * 16,
            'fp32_sweep': mv(8) + (20 if persistent else 33) * n * 8,
            'fp32_sweep_form': 'persistent launch' if persistent else 'graph of passes',
            'formula': '#matvecs * (N(8W+2w_v) + P w_v + M(8W+w_c) + 8WJ) + #vector passes * N w_v'}


def locg_times(rq, op, wl, dev, use_graph=True):
    """Time-to-E0 of the FP64 path (reference algorithm) and of the mixed-precision path."""
    import torch
    x0 = torch.as_tensor(wl.start_vector(np.complex128), device=dev)
    # tol=None: the reference default (dtype epsilon in its N-scaled test, ground_locg.py:
    # 224-225, 371-376), i.e. a converged FP64 energy to compare the mixed path against.
    res = {'start_vector': 'complex128 N(0,1)+iN(0,1), normalised', 'tol': None,
           'timing': 'median of 3 solves per mode after one warm-up solve',
           'cuda_graphs': use_graph}
    for mode in ('fp64', 'mixed'):
        rq.ground_locg(op, x0, mode=mode, use_graph=use_graph)   # warm-up: a whole solve
        runs = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e, vec, it = rq.ground_locg(op, x0, mode=mode, use_graph=use_graph)
            torch.cuda.synchronize()
            runs.append(time.perf_counter() - t0)
        res[mode] = {'time_to_e0_s': statistics.median(runs), 'runs_s': runs, 'eigval': e,
                     'niter': it, 'residual': rq.ground_locg.last_residual}
    e64 = res['fp64']['eigval']
    res['mixed']['rel_err_vs_fp64'] = abs(res['mixed']['eigval'] - e64) / abs(e64)
    res['speedup_mixed_vs_fp64'] = res['fp64']['time_to_e0_s'] / res['mixed']['time_to_e0_s']
    return res


def run_batched(args):
    """C4: 96 16-orbital JW instances (own seeds, a_i x b_i product subspaces).  Times the
    sequential per-instance FP64 solver loop and the batched mixed-precision solver, each from
    operator construction to energies, and reports instances/s."""
    import torch
    torch.cuda.set_device(0)
    import rqutils_b200 as rq
    from rqutils_b200 import workloads as W, _lib
    from rqutils_b200.batched import solve_instances
    t0 = time.perf_counter()
    structure = W.JWStructure(16)
    instances = W.c4(0, structure=structure)
    gen_s = time.perf_counter() - t0
    count = len(instances)

    def seq_fp64():
        e = np.zeros(count)
        it = np.zeros(count, dtype=np.int64)
        for i, w in enumerate(instances):
            ham = rq.PauliSumXZ.from_xz(w.x, w.z, w.coeffs, 32, force_real=True, padded=True)
            op = rq.SQDOperator(ham, rq.Subspace.from_u64(w.states, 32), cache_strategy=(1, 2))
            e[i], _, it[i] = rq.ground_locg(op, op.vinit(), vspace=(op.size, torch.complex128))
            big = op.nnz > 1e9
            del op, ham
            if big:
                _lib.trim_memory()
        return e, it

    res = {}
    for name, fn in (('batched_mixed', lambda: solve_instances(instances)),
                     ('sequential_fp64', seq_fp64)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        e, it = fn()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
        _lib.trim_memory()
        res[name] = {'time_s': dt, 'instances_per_s': count / dt, 'eigvals': e.tolist(),
                     'niter_total': int(it.sum())}
    e_b = np.array(res['batched_mixed']['eigvals'])
    e_s = np.array(res['sequential_fp64']['eigvals'])
    rel = np.abs(e_b - e_s) / np.abs(e_s)
    a, b = W.c4_dims(0)
    line = {'metric': 'C4 instances/s (96 JW instances, batched mixed vs sequential FP64)',
            'value': res['batched_mixed']['instances_per_s'], 'unit': 'instances/s',
            'higher_is_better': True, 'n_gpus': 1, 'dtype': 'complex128 results',
            'data': 'synthetic (seeded generator)',
            'config': {'workload': 'c4: 96 x (16-orbital JW, a_i x b_i 4-electron strings)',
                       'rows_total': int(sum(w.states.shape[0] for w in instances)),
                       'a': a.tolist(), 'b': b.tolist(), 'generation_s': gen_s},
            'sequential_fp64': {k: v for k, v in res['sequential_fp64'].items()
                                if k != 'eigvals'},
            'batched_mixed': {k: v for k, v in res['batched_mixed'].items() if k != 'eigvals'},
            'speedup': res['sequential_fp64']['time_s'] / res['batched_mixed']['time_s'],
            'max_rel_energy_diff': float(rel.max()), 'median_rel_energy_diff': float(np.median(rel))}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == 'reference':
        run_reference(args)
    elif args.workload == 'c4':
        run_batched(args)
    else:
        run_ours(args)


if __name__ == '__main__':
    main()
