"""``jax.numpy`` of the NumPy stand-in (test infrastructure only).

Every function forwards to NumPy with JAX-only keyword arguments (``out_sharding``) dropped and
array results returned as ``Array``.  Functions whose JAX semantics differ from NumPy's are
written out: ``bincount`` with ``length`` (negative values count as 0, values at or above
``length`` are dropped), ``array``/``asarray`` (always a new value).
"""
import types

import numpy as _np

from ._core import Array, wrap as _wrap, tree_map as _tree_map

ndarray = Array
integer = _np.integer
inexact = _np.inexact
floating = _np.floating
complexfloating = _np.complexfloating
float32, float64 = _np.float32, _np.float64
complex64, complex128 = _np.complex64, _np.complex128
int32, int64, uint8, uint32, uint64 = _np.int32, _np.int64, _np.uint8, _np.uint32, _np.uint64
bool_ = _np.bool_
inf, nan, pi = _np.inf, _np.nan, _np.pi
finfo, iinfo, issubdtype, dtype = _np.finfo, _np.iinfo, _np.issubdtype, _np.dtype


def _result(value):
    return _tree_map(_wrap, value)


def _forward(fn):
    def call(*args, **kwargs):
        kwargs.pop('out_sharding', None)
        kwargs.pop('device', None)
        return _result(fn(*args, **kwargs))
    call.__name__ = getattr(fn, '__name__', 'fn')
    return call


def bincount(x, weights=None, minlength=0, *, length=None):
    x = _np.asarray(x)
    if length is None:
        length = max(int(minlength), int(x.max()) + 1 if x.size else 0)
    x = _np.clip(x, 0, None)
    keep = x < length
    w = None if weights is None else _np.asarray(weights)[keep]
    return _wrap(_np.bincount(x[keep], weights=w, minlength=length)[:length])


def asarray(a, dtype=None, **kw):
    return _wrap(_np.array(a, dtype=dtype))


def array(a, dtype=None, **kw):
    return _wrap(_np.array(a, dtype=dtype))


def atan2(y, x):
    return _result(_np.arctan2(y, x))


def __getattr__(name):
    fn = getattr(_np, name)
    if callable(fn):
        return _forward(fn)
    return fn


linalg = types.SimpleNamespace(norm=_forward(_np.linalg.norm),
                               eigh=_forward(_np.linalg.eigh))
