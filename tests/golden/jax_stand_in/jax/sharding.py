"""``jax.sharding`` of the NumPy stand-in: one device, an empty abstract mesh."""


class PartitionSpec(tuple):
    def __new__(cls, *parts):
        return super().__new__(cls, parts)


class _Mesh:
    empty = True
    size = 1
    axis_names = ()
    shape = {}


_EMPTY_MESH = _Mesh()


class NamedSharding:
    def __init__(self, mesh, spec):
        self.mesh = mesh
        self.spec = spec


def get_abstract_mesh():
    return _EMPTY_MESH
