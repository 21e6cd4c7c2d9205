"""``jax.lax`` of the NumPy stand-in (test infrastructure only).

Control flow runs as Python loops; ``sort`` is a stable lexicographic sort over the first
``num_keys`` operands (``jax.lax.sort`` defaults to ``is_stable=True``); ``cond`` returns its
branch's outputs as arrays, as JAX does.
"""
import enum

import numpy as np

from ._core import wrap, to_array, tree_map, tree_leaves


class Precision(enum.Enum):
    DEFAULT = 0
    HIGH = 1
    HIGHEST = 2


def sort(operand, dimension=-1, is_stable=True, num_keys=1):
    single = not isinstance(operand, (tuple, list))
    ops = [np.asarray(operand)] if single else [np.asarray(o) for o in operand]
    if ops[0].ndim != 1:
        raise NotImplementedError('the stand-in sorts 1-D operands')
    keys = ops[:num_keys]
    perm = np.lexsort(tuple(keys[::-1]))          # lexsort: last key is primary; stable
    out = tuple(wrap(np.array(o[perm])) for o in ops)
    return out[0] if single else out


def ne(a, b):
    return wrap(np.asarray(np.not_equal(a, b)))


def iota(dtype, size, **kw):
    return wrap(np.arange(size, dtype=dtype))


def broadcasted_iota(dtype, shape, dimension, out_sharding=None, **kw):
    shape = tuple(shape)
    r = np.arange(shape[dimension], dtype=dtype)
    view = [1] * len(shape)
    view[dimension] = shape[dimension]
    return wrap(np.array(np.broadcast_to(r.reshape(view), shape)))


def dot(a, b, precision=None, preferred_element_type=None, out_sharding=None):
    return wrap(np.asarray(np.dot(a, b)))


def scan(f, init, xs=None, length=None, reverse=False, unroll=1):
    leaves = tree_leaves(xs) if xs is not None else []
    n = length if not leaves else np.asarray(leaves[0]).shape[0]
    carry = init
    ys = []
    order = range(n - 1, -1, -1) if reverse else range(n)
    for i in order:
        x_i = (tree_map(lambda a: wrap(np.asarray(a)[i]) if np.ndim(np.asarray(a)[i]) else
                        np.asarray(a)[i], xs) if xs is not None else None)
        carry, y = f(carry, x_i)
        ys.append(y)
    if reverse:
        ys = ys[::-1]
    if not ys or all(y is None for y in ys):
        stacked = None
    else:
        stacked = tree_map(lambda *parts: wrap(np.stack([np.asarray(p) for p in parts])),
                           ys[0], *ys[1:])
    return carry, stacked


def while_loop(cond_fun, body_fun, init_val):
    val = init_val
    while bool(cond_fun(val)):
        val = body_fun(val)
    return val


def fori_loop(lower, upper, body_fun, init_val):
    val = init_val
    for i in range(int(lower), int(upper)):
        val = body_fun(i, val)
    return val


def _aval(leaf):
    """(shape, dtype) of a branch output; None for a Python scalar (weakly typed in JAX, so it
    takes the other branch's dtype)."""
    if isinstance(leaf, (bool, int, float, complex)):
        return None
    a = np.asarray(leaf)
    return a.shape, a.dtype


def cond(pred, true_fun, false_fun, *operands):
    """JAX traces both branches and raises TypeError unless their outputs have identical
    structure, shapes and dtypes (weakly typed Python scalars excepted); the stand-in evaluates
    both (they are pure) to apply the same check, then returns the taken branch's outputs."""
    with np.errstate(all='ignore'):
        outs = (true_fun(*operands), false_fun(*operands))
    leaves = [tree_leaves(o) for o in outs]
    if len(leaves[0]) != len(leaves[1]):
        raise TypeError('true_fun and false_fun output must have identical types')
    for a, b in zip(*leaves):
        va, vb = _aval(a), _aval(b)
        if va is not None and vb is not None and va != vb:
            raise TypeError('true_fun and false_fun output must have identical types, got '
                            f'{va} and {vb}')
    return tree_map(to_array, outs[0] if bool(pred) else outs[1])


def map(f, xs):
    return scan(lambda _, x: (None, f(x)), None, xs)[1]


def pcast(x, axes, to=None):
    return x
