"""NumPy stand-in for the parts of `jax` the reference barotropic path imports.

Test infrastructure only: ``tests/golden/make_golden.py`` puts this directory
first on ``sys.path`` so that the reference's own hot-path modules
(src/licom/momentum/barotr*.py, src/licom/operators/*.py,
src/licom/kernel/{cube,communication}.py) run unmodified on the CPU in float64
with single-device (pdev = px = py = 1) semantics.  It implements exactly the
API surface those modules use; nothing here is shipped or imported by the
package.
"""
from . import numpy, lax, sharding  # noqa: F401
from .numpy import Arr


def jit(fn=None, **kwargs):
    if fn is None:
        return lambda f: f
    return fn


def _take(x, axis, k):
    return Arr._wrap(numpy.asnp(x).take(k, axis=axis))


def vmap(fn, in_axes=0, out_axes=0):
    """Loop-and-stack vmap (enough for cube_rmp's in_axes=(1, None, ...))."""
    def wrapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        size = None
        for a, ax in zip(args, axes):
            if ax is not None:
                size = numpy.asnp(a).shape[ax]
                break
        outs = []
        for k in range(size):
            sub = [(_take(a, ax, k) if ax is not None else a) for a, ax in zip(args, axes)]
            outs.append(fn(*sub))
        if isinstance(outs[0], tuple):
            return tuple(numpy.stack([o[i] for o in outs], axis=out_axes)
                         for i in range(len(outs[0])))
        return numpy.stack(outs, axis=out_axes)
    return wrapped


class _TreeUtil:
    @staticmethod
    def tree_map(f, tree):
        if isinstance(tree, (tuple, list)):
            return type(tree)(f(t) for t in tree)
        return f(tree)


tree_util = _TreeUtil()


def device_put(x, *a, **k):
    return x


def device_get(x):
    return x
