"""Array type and tree helpers of the NumPy stand-in for JAX (test infrastructure only).

``Array`` is an ``ndarray`` subclass with JAX's value semantics where NumPy's differ:

* in-place operators (``a -= b``) rebind instead of writing into ``a``, because JAX arrays are
  immutable and code written for JAX may hold other references to ``a``;
* reading ``a[i]`` with an out-of-bound integer index returns the clamped element, as JAX's
  gather does, where NumPy raises;
* ``a.at[idx].get/set/add/subtract/multiply`` return new arrays with JAX's index rules:
  negative indices wrap unless ``wrap_negative_indices=False``; out-of-bound gathers return
  ``fill_value`` in ``mode='fill'`` and are clamped otherwise; out-of-bound scatters are dropped;
  scatter updates are cast to the array's dtype; ``add`` accumulates repeated indices.
"""
import dataclasses

import numpy as np


def _clamp_one(i, n):
    if isinstance(i, (bool, np.bool_)):
        return i
    if isinstance(i, (int, np.integer)):
        i = int(i)
        if i < 0:
            i += n
        return min(max(i, 0), n - 1) if n > 0 else i
    if isinstance(i, np.ndarray) and np.issubdtype(i.dtype, np.integer):
        j = np.where(i < 0, i + n, i)
        return np.clip(j, 0, n - 1) if n > 0 else j
    return i


def _clamp_index(idx, shape):
    if isinstance(idx, tuple):
        if any(i is Ellipsis or i is None for i in idx):
            return idx
        return tuple(_clamp_one(i, shape[a]) if a < len(shape) else i
                     for a, i in enumerate(idx))
    if len(shape) == 0:
        return idx
    return _clamp_one(idx, shape[0])


class Array(np.ndarray):
    """ndarray with JAX's immutable-value semantics (see module docstring)."""

    def __array_finalize__(self, obj):
        pass

    def __getitem__(self, idx):
        return super().__getitem__(_clamp_index(idx, self.shape))

    def __iter__(self):
        # iteration must stop at the end, which clamped indexing alone would never signal
        if self.ndim == 0:
            raise TypeError('iteration over a 0-d array')
        for i in range(self.shape[0]):
            yield super().__getitem__(i)

    @property
    def at(self):
        return _At(self)

    # functional in-place operators: ``a op= b`` evaluates ``a op b`` and rebinds the name
    def __iadd__(self, o):
        return np.add(self, o)

    def __isub__(self, o):
        return np.subtract(self, o)

    def __imul__(self, o):
        return np.multiply(self, o)

    def __itruediv__(self, o):
        return np.true_divide(self, o)

    def __ifloordiv__(self, o):
        return np.floor_divide(self, o)

    def __imod__(self, o):
        return np.mod(self, o)

    def __ipow__(self, o):
        return np.power(self, o)

    def __iand__(self, o):
        return np.bitwise_and(self, o)

    def __ior__(self, o):
        return np.bitwise_or(self, o)

    def __ixor__(self, o):
        return np.bitwise_xor(self, o)

    def __ilshift__(self, o):
        return np.left_shift(self, o)

    def __irshift__(self, o):
        return np.right_shift(self, o)


def wrap(value):
    """ndarray -> Array (no copy); scalars and other objects unchanged."""
    if isinstance(value, np.ndarray) and not isinstance(value, Array):
        return value.view(Array)
    return value


def to_array(value):
    """Like ``jnp.asarray`` for leaves: Python and NumPy scalars become 0-d arrays."""
    if isinstance(value, Array):
        return value
    if isinstance(value, (np.ndarray, np.generic, bool, int, float, complex)):
        return np.asarray(value).view(Array)
    return value


def tree_map(fn, tree, *rest, is_leaf=None):
    """Map over tuples, lists, dicts, dataclasses (static fields skipped) and leaves."""
    if is_leaf is not None and is_leaf(tree):
        return fn(tree, *rest)
    if tree is None:
        return None
    if isinstance(tree, tuple) and not hasattr(tree, '_fields'):
        return tuple(tree_map(fn, t, *(r[i] for r in rest), is_leaf=is_leaf)
                     for i, t in enumerate(tree))
    if isinstance(tree, list):
        return [tree_map(fn, t, *(r[i] for r in rest), is_leaf=is_leaf)
                for i, t in enumerate(tree)]
    if isinstance(tree, dict):
        return {k: tree_map(fn, v, *(r[k] for r in rest), is_leaf=is_leaf)
                for k, v in tree.items()}
    if dataclasses.is_dataclass(tree) and not isinstance(tree, type):
        changes = {}
        for f in dataclasses.fields(tree):
            if f.metadata.get('static', False):
                continue
            changes[f.name] = tree_map(fn, getattr(tree, f.name),
                                       *(getattr(r, f.name) for r in rest), is_leaf=is_leaf)
        return dataclasses.replace(tree, **changes)
    return fn(tree, *rest)


def tree_leaves(tree):
    out = []
    tree_map(lambda a: out.append(a), tree)
    return out


def _is_int_array(idx):
    return isinstance(idx, np.ndarray) and np.issubdtype(idx.dtype, np.integer)


def _normalise(idx, n, wrap_negative):
    idx = np.asarray(idx).astype(np.int64)
    if wrap_negative:
        idx = np.where(idx < 0, idx + n, idx)
    return idx


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIndex(self.arr, idx)


class _AtIndex:
    def __init__(self, arr, idx):
        self.arr = arr
        self.idx = idx

    # gathers ---------------------------------------------------------------------------------
    def get(self, *, mode=None, fill_value=None, wrap_negative_indices=True, out_sharding=None,
            indices_are_sorted=False, unique_indices=False):
        arr, idx = self.arr, self.idx
        if not _is_int_array(idx):
            out = arr[idx]
            return wrap(np.array(out)) if isinstance(out, np.ndarray) else out
        n = arr.shape[0]
        pos = _normalise(idx, n, wrap_negative_indices)
        inb = (pos >= 0) & (pos < n)
        base = np.asarray(arr)
        if mode == 'fill':
            if fill_value is None:
                fill_value = np.nan if np.issubdtype(arr.dtype, np.inexact) else 0
            out = np.full(pos.shape + arr.shape[1:], fill_value, dtype=arr.dtype)
            out[inb] = base[pos[inb]]
            return wrap(out)
        return wrap(np.array(base[np.clip(pos, 0, n - 1)]))

    # scatters --------------------------------------------------------------------------------
    def _scatter(self, values, op, wrap_negative_indices=True):
        arr = np.array(self.arr)                      # copy: the result is a new value
        values = np.asarray(values).astype(arr.dtype)
        idx = self.idx
        if _is_int_array(idx):
            n = arr.shape[0]
            pos = _normalise(idx, n, wrap_negative_indices)
            inb = (pos >= 0) & (pos < n)              # out-of-bound updates are dropped
            if values.ndim and values.shape[:pos.ndim] == pos.shape:
                values = values[inb]
            pos = pos[inb]
            if op == 'set':
                arr[pos] = values
            elif op == 'add':
                np.add.at(arr, pos, values)
            elif op == 'mul':
                np.multiply.at(arr, pos, values)
            return wrap(arr)
        if op == 'set':
            arr[idx] = values
        elif op == 'add':
            arr[idx] = arr[idx] + values
        elif op == 'mul':
            arr[idx] = arr[idx] * values
        return wrap(arr)

    def set(self, values, *, mode=None, wrap_negative_indices=True, out_sharding=None,
            indices_are_sorted=False, unique_indices=False):
        return self._scatter(values, 'set', wrap_negative_indices)

    def add(self, values, *, mode=None, wrap_negative_indices=True, out_sharding=None,
            indices_are_sorted=False, unique_indices=False):
        return self._scatter(values, 'add', wrap_negative_indices)

    def subtract(self, values, **kw):
        return self.add(-np.asarray(values), **kw)

    def multiply(self, values, *, mode=None, wrap_negative_indices=True, out_sharding=None,
                 indices_are_sorted=False, unique_indices=False):
        return self._scatter(values, 'mul', wrap_negative_indices)
