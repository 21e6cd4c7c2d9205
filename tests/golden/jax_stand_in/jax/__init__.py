"""NumPy stand-in for the JAX subset used by rqutils' SQD path (test infrastructure only).

Single device, ``jax_enable_x64`` semantics.  ``jit`` converts its non-static arguments to
arrays (as JAX traces them) and calls the function eagerly; the sharding API answers for an
empty mesh; ``debug.print`` formats and prints like JAX's (a format string is required).
"""
import functools
import inspect
import types

import numpy as _np

from . import numpy, lax, sharding, tree_util          # noqa: F401  (attributes of jax)
from ._core import Array, tree_map as _tree_map, to_array as _to_array

__version__ = '0.0-numpy-stand-in'


def jit(fun=None, *, static_argnames=(), static_argnums=(), donate_argnums=(), **kw):
    if fun is None:
        return lambda f: jit(f, static_argnames=static_argnames, static_argnums=static_argnums)
    if isinstance(static_argnames, str):
        static_argnames = (static_argnames,)
    static_argnames = set(static_argnames)
    static_argnums = {static_argnums} if isinstance(static_argnums, int) else set(static_argnums)
    sig = inspect.signature(fun)

    @functools.wraps(fun)
    def call(*args, **kwargs):
        bound = sig.bind(*args, **kwargs)
        for i, (name, value) in enumerate(list(bound.arguments.items())):
            param = sig.parameters[name]
            if name in static_argnames or i in static_argnums:
                continue
            if param.kind == inspect.Parameter.VAR_POSITIONAL:
                bound.arguments[name] = tuple(_tree_map(_to_array, v) for v in value)
            else:
                bound.arguments[name] = _tree_map(_to_array, value)
        return fun(*bound.args, **bound.kwargs)
    return call


class _Aval:
    def __init__(self, x):
        self.shape = _np.shape(x)
        self.dtype = _np.asarray(x).dtype
        self.sharding = sharding.NamedSharding(sharding._EMPTY_MESH,
                                               sharding.PartitionSpec(*([None] * len(self.shape))))
        self.manual_axis_type = types.SimpleNamespace(varying=frozenset())


def typeof(x):
    return _Aval(x)


def reshard(x, spec):
    raise NotImplementedError('the stand-in has one device: no resharding')


def shard_map(*a, **k):
    raise NotImplementedError('the stand-in has one device: no shard_map')


def _print(fmt=None, *args, ordered=False, **kwargs):
    if fmt is None:
        raise TypeError("print() missing 1 required positional argument: 'fmt'")
    print(fmt.format(*args, **kwargs), flush=True)


debug = types.SimpleNamespace(print=_print)
tree = types.SimpleNamespace(map=lambda f, *trees, **k: _tree_map(f, *trees),
                             leaves=tree_util.tree_leaves)
