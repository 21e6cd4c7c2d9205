"""Host-side logic of bench.py that needs no GPU: traffic lookup per layout, the LOCG byte
formula, workload naming."""
import bench


def _profiles(tmp_path, files):
    (tmp_path / 'profiles').mkdir()
    for name, text in files.items():
        (tmp_path / 'profiles' / name).write_text(text)


def test_traffic_follows_the_chosen_layout_and_current_sources(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, 'ROOT', str(tmp_path))
    monkeypatch.setattr(bench, 'kernel_sources_digest', lambda: 'abc')
    _profiles(tmp_path, {
        'matvec_c2_cache12.md': 'traffic_bytes_per_launch: 300\nkernel_sources_sha256: abc\n',
        'matvec_c2_cache12_product-csr.md':
            'x\ntraffic_bytes_per_launch: 200\nkernel_sources_sha256: abc\n',
        'matvec_c3_cache12_product.md': 'traffic_bytes_per_launch: 9\nkernel_sources_sha256: old\n',
    })
    assert bench.load_traffic('c2', (1, 2), 'csr')[0] == 300
    assert bench.load_traffic('c2', (1, 2), 'product-csr')[0] == 200
    # the product layout falls back to the other product summary
    assert bench.load_traffic('c2', (1, 2), 'product')[0] == 200
    # a capture of other kernel sources is not used
    val, note = bench.load_traffic('c3', (1, 2), 'product')
    assert val is None and 'other kernel sources' in note
    assert bench.load_traffic('c1', (1, 2), 'csr')[0] is None
    # FP32 vectors use their own summaries
    assert bench.load_traffic('c2', (1, 2), 'product-csr', 'fp32')[0] is None


def test_kernel_sources_digest_is_stable():
    assert bench.kernel_sources_digest() == bench.kernel_sources_digest()
    assert len(bench.kernel_sources_digest()) == 64


def test_cpu_sample_is_shared_and_seeded():
    wl = bench.make_workload('c1')
    a = bench.cpu_sample(wl)
    b = bench.cpu_sample(wl)
    assert (a == b).all() and a.shape[0] == 2000 and (a[1:] > a[:-1]).all()
    assert bench.cpu_sample(wl, rows=100).shape[0] == 100


def test_locg_bytes_formula():
    n, m, j, p = 262144, 94849, 18281, 115178144
    b = bench.locg_bytes(n, m, j, p)
    mv64 = n * (8 + 32) + p * 16 + m * 24 + j * 8
    mv32 = n * (8 + 16) + p * 8 + m * 24 + j * 8
    assert b['fp64'] == 4 * mv64 + 42 * n * 16
    assert b['fp32_sweep'] == mv32 + 33 * n * 8
    # the matvec part is the roofline formula the bench reports for C2 (1.856 GB)
    assert mv64 == 1855758688


def test_workload_names_and_configs():
    wl = bench.make_workload('c1')
    cfg = bench.workload_config(wl, (1, 2))
    assert cfg['subspace_dim'] == 2000 and cfg['num_qubits'] == 16
    assert 'random Pauli sum' in cfg['workload']


def test_issue_bound_estimate():
    # C3 shape: the reference's on-the-fly diagonals would be popcount-bound at ~1.75 s per
    # matvec, the cached FP64 elements need well under the measured 6 ms of FP64 FMAs
    n, m, p = 16777216, 485281, 2653787580
    b = bench.issue_bound(n, m, p, False, 148, 1965.0, 6.0e-3)
    assert b['reference_popcounts_per_matvec'] == n * m
    assert abs(b['reference_popcount_floor_ms'] - n * m / (16 * 148 * 1965e6) * 1e3) < 1e-9
    assert 1500 < b['reference_popcount_floor_ms'] < 2000
    assert b['cached_fp64_fma_per_matvec'] == 2 * p
    assert b['cached_fp64_fma_floor_ms'] < 0.1 * b['timed_matvec_ms']
    assert bench.issue_bound(n, m, p, True, 148, 1965.0, 6.0e-3)['cached_fp64_fma_per_matvec'] \
        == 4 * p
