"""Host-side logic that needs no GPU: argument validation with the reference's error behaviour,
option handling, layout conversions, and the absence of a CPU fallback."""
import numpy as np
import pytest
import torch

import rqutils_b200 as rq
from rqutils_b200 import _lib, workloads as W
from rqutils_b200.paulis.symplectic import _pack_masks, _unpack_masks
from oracle import symplectic as OS


def test_from_paulisum_validation_matches_reference():
    with pytest.raises(ValueError, match='Lengths of Pauli and coeff lists'):
        rq.PauliSumXZ.from_paulisum((['XX', 'ZZ'], [1.0]))
    with pytest.raises(ValueError, match='non-uniform lengths'):
        rq.PauliSumXZ.from_paulisum((['XX', 'ZZZ'], [1.0, 2.0]))
    with pytest.raises(ValueError, match='Unsupported input type'):
        rq.PauliSumXZ.from_paulisum({'XX': 1.0})


def test_sqd_states_size_validation():
    with pytest.raises(ValueError, match='states_size smaller'):
        rq.sqd((['ZZ'], [1.0]), np.zeros((4, 2), dtype=np.uint8), states_size=3)


def test_options_from_dict_and_defaults_match_reference():
    opts = rq.SQDOptions(**{'return_eigvec': False, 'locg_tol': 1e-9})
    assert opts.cache_strategy == (1, 0)
    assert opts.shard_bundle == 1
    assert opts.locg_maxiter == 1000
    assert opts.return_eigvec is False and opts.locg_tol == 1e-9


def test_mask_packing_matches_reference_layout():
    rng = np.random.default_rng(0)
    x, z, c = W.random_pauli_sum(11, 30, rng)
    labels = W.labels_from_xz(x, z, 11)
    ref = OS.from_paulisum((labels, list(c)), add_padding=True)
    # unpack the reference's packed X signatures and repack them
    masks = _unpack_masks(ref.x, 11, True)
    assert (_pack_masks(masks, 11, True) == ref.x).all()
    assert (np.sort(masks) == masks).all()   # groups ascending in x


@pytest.mark.skipif(torch.cuda.is_available(), reason='checks the no-GPU behaviour')
def test_no_cpu_fallback():
    with pytest.raises(_lib.SQDError, match='no CPU fallback'):
        rq.PauliSumXZ.from_paulisum((['XX', 'ZZ'], [1.0, 2.0]))
    with pytest.raises(_lib.SQDError):
        rq.Subspace.from_bits(np.zeros((3, 2), dtype=np.uint8))


def test_workload_generators_are_seeded_and_shaped():
    a, b = W.c1(0), W.c1(0)
    assert (a.states == b.states).all() and (a.coeffs == b.coeffs).all()
    assert a.states.shape[0] == 2000
    assert all(bin(int(s)).count('1') == 8 for s in a.states[:50])
    st = W.product_subspace(6, 2, 5, 4, np.random.default_rng(1))
    assert st.shape[0] == 20 and (np.diff(st.astype(np.float64)) > 0).all()
    aa, bb = W.c4_dims(0)
    assert aa.shape == (96,) and aa.min() >= 64 and bb.max() <= 1820


def test_every_package_module_imports():
    """Lazily imported modules (autotune, autograd, batched, ...) must at least import."""
    import importlib
    import pkgutil
    import rqutils_b200
    names = [m.name for m in pkgutil.walk_packages(rqutils_b200.__path__, 'rqutils_b200.')]
    assert 'rqutils_b200.autotune' in names
    for name in names:
        importlib.import_module(name)


@pytest.mark.parametrize('norb', [3, 5])
def test_jw_structure_map_reproduces_the_jw_hamiltonian(norb):
    """The batched workload's shortcut (a fixed sparse map from the independent integrals to the
    Pauli coefficients) gives the same Pauli sum as the direct Jordan-Wigner construction."""
    from rqutils_b200 import workloads as W
    rng = np.random.default_rng(40 + norb)
    h1, h2 = W.random_integrals(norb, rng)
    st = W.JWStructure(norb)

    def as_dict(x, z, c):
        d = {}
        for xi, zi, ci in zip(np.asarray(x, np.uint64), np.asarray(z, np.uint64), np.asarray(c)):
            d[(int(xi), int(zi))] = d.get((int(xi), int(zi)), 0.0) + complex(ci)
        return {k: v for k, v in d.items() if abs(v) > 1e-12}

    direct = as_dict(*W.jw_hamiltonian(h1, h2))
    mapped = as_dict(*st.hamiltonian(h1, h2))
    assert direct.keys() == mapped.keys()
    scale = max(abs(v) for v in direct.values())
    assert max(abs(direct[k] - mapped[k]) for k in direct) <= 1e-13 * scale
