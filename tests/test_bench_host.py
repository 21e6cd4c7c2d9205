"""Host-side logic of bench.py that needs no GPU: traffic lookup per layout, the LOCG byte
formula, workload naming."""
import bench


def test_traffic_follows_the_chosen_layout():
    csr = bench.load_traffic('c2', (1, 2), 'csr')
    prod_csr = bench.load_traffic('c2', (1, 2), 'product-csr')
    prod = bench.load_traffic('c2', (1, 2), 'product')
    assert csr is not None and prod_csr is not None
    assert prod_csr < csr                 # the slabs read fewer bytes than the pair lists
    assert prod == prod_csr               # falls back to the other product summary
    assert bench.load_traffic('c3', (1, 2), 'product') > 1e10
    assert bench.load_traffic('c1', (1, 2), 'csr') is None


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


def test_fp32_traffic_uses_its_own_summaries():
    assert bench.load_traffic('c2', (1, 2), 'product-csr', 'fp32') is None
    assert bench.load_traffic('c2', (1, 2), 'product-csr', 'fp64') is not None
