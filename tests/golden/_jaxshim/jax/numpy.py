"""NumPy-backed `jax.numpy` subset with functional ``.at[...]`` updates."""
import numpy as _np

int32 = _np.int32
float64 = _np.float64
float32 = _np.float32
s_ = _np.s_
ndarray = _np.ndarray


def asnp(x):
    return _np.asarray(x).view(_np.ndarray) if isinstance(x, _np.ndarray) else _np.asarray(x)


class _AtIndexer:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def set(self, v):
        out = _np.array(asnp(self._arr), copy=True)
        out[self._idx] = asnp(v)
        return Arr._wrap(out)

    def add(self, v):
        out = _np.array(asnp(self._arr), copy=True)
        out[self._idx] += asnp(v)
        return Arr._wrap(out)


class _At:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtIndexer(self._arr, idx)


class Arr(_np.ndarray):
    """ndarray subclass carrying JAX's functional ``.at[idx].set/.add``."""

    @staticmethod
    def _wrap(x):
        x = _np.asarray(x)
        return x.view(Arr)

    @property
    def at(self):
        return _At(self)


def _w(fn):
    def g(*a, **k):
        return Arr._wrap(fn(*a, **k))
    g.__name__ = fn.__name__
    return g


def array(x, dtype=None):
    return Arr._wrap(_np.array(asnp(x) if isinstance(x, _np.ndarray) else x, dtype=dtype))


asarray = array


def pad(x, pad_width, mode="constant", constant_values=0):
    return Arr._wrap(_np.pad(asnp(x), pad_width, mode=mode, constant_values=constant_values))


def where(c, a, b):
    return Arr._wrap(_np.where(asnp(c), asnp(a), asnp(b)))


def stack(xs, axis=0):
    return Arr._wrap(_np.stack([asnp(x) for x in xs], axis=axis))


maximum = _w(_np.maximum)
minimum = _w(_np.minimum)
sqrt = _w(_np.sqrt)
sin = _w(_np.sin)
cos = _w(_np.cos)
swapaxes = _w(_np.swapaxes)
flip = _w(_np.flip)
expand_dims = _w(_np.expand_dims)
take_along_axis = _w(_np.take_along_axis)
arange = _w(_np.arange)
zeros = _w(_np.zeros)
ones = _w(_np.ones)
zeros_like = _w(_np.zeros_like)
ones_like = _w(_np.ones_like)
transpose = _w(_np.transpose)
reshape = _w(_np.reshape)
