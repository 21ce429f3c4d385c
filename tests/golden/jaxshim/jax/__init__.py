"""NumPy stand-in for jax (golden-vector generation only; see _core.py)."""
from __future__ import annotations

import numpy as _np

from . import _core
from . import numpy as numpy  # noqa: F401
from . import lax, tree_util, tree, debug, scipy, flatten_util  # noqa: F401

Array = _np.ndarray
vmap = _core.vmap


class _Config:
    def __init__(self):
        self._v = {"jax_enable_x64": True}

    def update(self, k, v):
        self._v[k] = v

    def read(self, k):
        return self._v.get(k)


config = _Config()


def jit(f=None, **kw):
    if f is None:
        return lambda g: g
    return f


def checkpoint(f=None, **kw):
    if f is None:
        return lambda g: g
    return f


remat = checkpoint


def block_until_ready(x):
    return x


def jvp(f, primals, tangents):
    """Forward derivative for the only use on the reference's static-geometry path:
    tangents that are all empty containers (no control surfaces) give zero tangents."""
    leaves, _ = _core.flatten(tangents)
    out = f(*primals)
    if leaves:
        raise NotImplementedError("jvp with non-empty tangents is not provided by the stand-in")
    return out, _core.tree_map(lambda a: _core.wrap(_np.zeros_like(a)), out)


def _unavailable(name):
    def f(*a, **k):
        raise NotImplementedError(f"jax.{name} is not provided by the NumPy stand-in")

    return f


vjp = _unavailable("vjp")
jacrev = _unavailable("jacrev")
jacfwd = _unavailable("jacfwd")
jacobian = _unavailable("jacobian")
linearize = _unavailable("linearize")
eval_shape = _unavailable("eval_shape")


class ShapeDtypeStruct:
    def __init__(self, shape, dtype):
        self.shape = shape
        self.dtype = dtype
