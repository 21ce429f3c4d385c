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


def _fd_step(primal_leaves, tangent_leaves):
    """Central-difference step for a directional derivative: 1e-6 of the inputs' scale
    along a unit tangent (truncation ~1e-12, rounding ~1e-10 relative)."""
    ps = max([float(_np.max(_np.abs(p))) for p in primal_leaves if _np.size(p)] + [1.0])
    ts = max([float(_np.max(_np.abs(t))) for t in tangent_leaves if _np.size(t)] + [0.0])
    return 0.0 if ts == 0.0 else 1e-6 * ps / ts


def jvp(f, primals, tangents):
    """Forward derivative by central differences of f along the tangents (the stand-in has
    no forward-mode AD); all-empty or all-zero tangents give zero tangents."""
    primals, tangents = tuple(primals), tuple(tangents)
    out = f(*primals)
    t_leaves, _ = _core.flatten(tangents)
    p_leaves, _ = _core.flatten(primals)
    h = _fd_step(p_leaves, t_leaves)
    if h == 0.0:
        return out, _core.tree_map(lambda a: _core.wrap(_np.zeros_like(_np.asarray(a, dtype=float))), out)
    shift = lambda s: tuple(_core.tree_map(lambda p, t: _core.wrap(_np.asarray(p) + s * _np.asarray(t)), p, t)
                            for p, t in zip(primals, tangents))
    fp, fm = f(*shift(h)), f(*shift(-h))
    tan = _core.tree_map(lambda a, b: _core.wrap((_np.asarray(a) - _np.asarray(b)) / (2.0 * h)), fp, fm)
    return out, tan


def jacobian(f, argnums=0, **_):
    """Jacobian of an array-valued f with respect to one array argument, column by column
    with the central differences of jvp; shape out.shape + x.shape."""
    if not isinstance(argnums, int):
        raise NotImplementedError("the stand-in's jacobian takes one argnum")

    def jac(*args):
        x = _np.asarray(args[argnums], dtype=float)
        cols = []
        for j in range(x.size):
            e = _np.zeros(x.size)
            e[j] = 1.0
            tangents = tuple(_core.tree_map(lambda a: _np.zeros_like(_np.asarray(a, dtype=float)), a)
                             if k != argnums else e.reshape(x.shape) for k, a in enumerate(args))
            _, t = jvp(f, args, tangents)
            cols.append(_np.asarray(t))
        out = _np.stack(cols, axis=-1)
        return _core.wrap(out.reshape(out.shape[:-1] + x.shape))

    return jac


jacfwd = jacobian


def _unavailable(name):
    def f(*a, **k):
        raise NotImplementedError(f"jax.{name} is not provided by the NumPy stand-in")

    return f


vjp = _unavailable("vjp")
jacrev = _unavailable("jacrev")
linearize = _unavailable("linearize")
eval_shape = _unavailable("eval_shape")


class ShapeDtypeStruct:
    def __init__(self, shape, dtype):
        self.shape = shape
        self.dtype = dtype
