"""Generates the golden fixtures in this folder (run: python -m tests.golden.make_golden).

The reference (rqutils, pure JAX) cannot run in this image (no jax) and ships no stored outputs,
so the fixtures hold the CPU oracle's outputs (a step-by-step restatement of the reference) on
small seeded inputs, each cross-checked here against the independent dense Kronecker-product
construction and numpy eigh before it is written.
"""
import os

import numpy as np

from rqutils_b200 import workloads as W
from oracle import symplectic as OS, sqd as OQ, dense as OD, ground_locg as OL

HERE = os.path.dirname(os.path.abspath(__file__))


def _labels_array(labels):
    return np.array([s.encode() for s in labels], dtype='S')


def paulis_small():
    rng = np.random.default_rng(101)
    x, z, c = W.random_pauli_sum(10, 80, rng)
    labels = W.labels_from_xz(x, z, 10)
    # explicit duplicates, a zero coefficient and a cancelling pair
    labels += [labels[3], labels[7], 'IIIIIIIIII', 'XYZIIIIIIZ', 'XYZIIIIIIZ']
    coeffs = np.concatenate([c, [0.5, -0.25, 1.5, 0.0, 2.0]])
    ham = OS.from_paulisum((labels, list(coeffs)), add_padding=True)
    cplx = coeffs + 1j * rng.standard_normal(coeffs.shape[0]) * 0.1
    hamc = OS.from_paulisum((labels, list(cplx)))
    return {'labels': _labels_array(labels), 'coeffs': coeffs, 'x': ham.x, 'z': ham.z,
            'c': ham.c, 'coeffs_complex': cplx, 'xc': hamc.x, 'zc': hamc.z, 'cc': hamc.c}


def sqd_small():
    rng = np.random.default_rng(202)
    n = 10
    x, z, c = W.random_pauli_sum(n, 60, rng)
    labels = W.labels_from_xz(x, z, n)
    uniq = W.weight_subspace(n, 5, 150, rng)
    # duplicates in the input, and fill-in slots (states_size > unique count)
    sample = np.concatenate([uniq, uniq[rng.integers(0, 150, size=40)]])
    rng.shuffle(sample)
    states = OQ.u64_to_states(sample, n)
    size = states.shape[0] + 7
    ham = OS.from_paulisum((labels, list(c)), force_real=True, add_padding=True)
    su = OQ.uniquify_states(OQ.pack_states(states), size)
    xsources = np.stack([OQ.get_xsource(xx, su) for xx in ham.x])
    diag0 = OQ.get_diagonal(ham.z[0], ham.c[0], su)
    v = rng.standard_normal(size) + 1j * rng.standard_normal(size)
    v[150:] = 0.0
    hv = OQ.apply_h_x_cached(v, xsources, ham.z, ham.c, su)
    vinit = OQ.vinit_index(ham, su)
    e_locg, vec, niter = OL.ground_locg(
        lambda vv: OQ.apply_h_x_cached(vv, xsources, ham.z, ham.c, su), vinit, tol=1e-12,
        vspace=(size, ham.c.dtype))
    h = OD.projected_matrix(labels, c, np.sort(uniq))
    e0 = np.linalg.eigvalsh(h)[0]
    assert abs(e_locg - e0) < 1e-9 * abs(e0)
    return {'labels': _labels_array(labels), 'coeffs': c, 'states': states,
            'states_size': np.array(size), 'states_u64': OQ.packed_to_u64(su[:150], n),
            'xsources': xsources, 'diag0': diag0, 'v': v, 'hv': hv, 'vinit': np.array(vinit),
            'eig_dense': np.array(e0), 'eig_locg': np.array(e_locg), 'niter': np.array(niter)}


def notebook_small():
    labels, coeffs, states = W.notebook_case(17, nq=12, nsample=2000, nterm=100)
    e, vec, basis = OQ.sqd((labels, list(coeffs)), states, options={'locg_tol': 1e-12})
    h = OD.projected_matrix(labels, coeffs, OQ.states_to_u64(basis))
    e0 = np.linalg.eigvalsh(h)[0]
    assert abs(e - e0) < 1e-8 * abs(e0)
    return {'labels': _labels_array(labels), 'coeffs': coeffs, 'states': states,
            'eig_dense': np.array(e0), 'eig_oracle': np.array(e)}


CASES = {'paulis_small': paulis_small, 'sqd_small': sqd_small, 'notebook_small': notebook_small}


def main():
    for name, fn in CASES.items():
        path = os.path.join(HERE, name + '.npz')
        np.savez_compressed(path, **fn())
        print('wrote', path, os.path.getsize(path))


if __name__ == '__main__':
    main()
