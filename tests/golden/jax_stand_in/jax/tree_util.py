"""``jax.tree_util`` of the NumPy stand-in."""
from ._core import tree_map, tree_leaves  # noqa: F401


def register_dataclass(cls=None, **kw):
    """Dataclass pytrees: the stand-in's tree helpers walk dataclass fields directly and skip
    fields whose metadata marks them static."""
    if cls is None:
        return lambda c: c
    return cls
