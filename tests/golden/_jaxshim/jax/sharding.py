"""`jax.sharding` stubs for a one-device mesh."""


class PartitionSpec(tuple):
    def __new__(cls, *args):
        return super().__new__(cls, args)


class Mesh:
    def __init__(self, devices=None, axis_names=("tile", "x", "y")):
        self.shape = {n: 1 for n in axis_names}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


class NamedSharding:
    def __init__(self, mesh, spec):
        self.mesh, self.spec = mesh, spec


class SingleDeviceSharding:
    def __init__(self, *a, **k):
        pass
