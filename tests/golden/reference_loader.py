"""Imports the UNMODIFIED reference modules (rqutils.sqd, rqutils.ground_locg,
rqutils.paulis.symplectic) from a reference checkout through the NumPy stand-in for JAX in
``jax_stand_in/`` (test infrastructure only; used by ``make_reference_golden.py`` in a container
that holds the reference checkout — the tests read only the fixtures it wrote).

The package ``__init__`` files of rqutils are not executed (``rqutils/__init__.py`` asks the
installed distribution for its version, and ``rqutils.paulis`` imports modules off the SQD path):
empty package objects whose ``__path__`` points into the checkout stand in for them, so the
three modules load from their own files exactly as shipped.
"""
import importlib
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
STAND_IN = os.path.join(HERE, 'jax_stand_in')


def _numpy_pad_accepts_dict():
    import numpy as np
    try:
        np.pad(np.zeros((1, 1)), {1: (1, 0)})
        return True
    except TypeError:
        return False


def _install_dict_pad():
    """The reference pads with ``np.pad(a, {axis: (before, after)})`` (symplectic.py:118-119,
    sqd.py:255), the per-axis dict form that NumPy accepts from 2.4 on; this image has NumPy
    2.3.  The same semantics (axes not named are not padded) come from a wrapper that expands
    the dict to NumPy's per-axis list before calling the real ``np.pad``."""
    import numpy as np
    real_pad = np.pad

    def pad(array, pad_width, mode='constant', **kwargs):
        if isinstance(pad_width, dict):
            widths = [(0, 0)] * np.ndim(array)
            for axis, w in pad_width.items():
                widths[axis] = (w, w) if np.isscalar(w) else tuple(w)
            pad_width = widths
        return real_pad(array, pad_width, mode, **kwargs)
    np.pad = pad


def load(reference_root):
    if not _numpy_pad_accepts_dict():
        _install_dict_pad()
    pkg_dir = os.path.join(reference_root, 'rqutils')
    if not os.path.isdir(pkg_dir):
        raise FileNotFoundError(f'no rqutils package under {reference_root}')
    if STAND_IN not in sys.path:
        sys.path.insert(0, STAND_IN)
    jax = importlib.import_module('jax')
    if not getattr(jax, '__version__', '').endswith('numpy-stand-in'):
        raise RuntimeError('a real jax is importable; the stand-in must not shadow it')
    for name, path in (('rqutils', pkg_dir), ('rqutils.paulis', os.path.join(pkg_dir, 'paulis'))):
        if name not in sys.modules:
            mod = types.ModuleType(name)
            mod.__path__ = [path]
            sys.modules[name] = mod
    symplectic = importlib.import_module('rqutils.paulis.symplectic')
    ground_locg = importlib.import_module('rqutils.ground_locg')
    sqd = importlib.import_module('rqutils.sqd')
    return types.SimpleNamespace(symplectic=symplectic, ground_locg=ground_locg, sqd=sqd)
