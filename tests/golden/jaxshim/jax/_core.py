"""A NumPy stand-in for the parts of ``jax`` that FLAPJAX's aero path uses.

Only for producing golden vectors from the reference source in a container without
JAX: arrays are float64 NumPy arrays with JAX's functional update syntax
(``a.at[i].set(v)``), transformations run eagerly (``vmap`` and ``lax.map`` loop and
stack, ``jit``/``checkpoint`` are the identity), and pytrees registered by the code under
test are flattened through a local registry.
"""
from __future__ import annotations

import numpy as np


class JArr(np.ndarray):
    """ndarray with JAX's immutable update and in-place-operator semantics."""

    def __array_finalize__(self, obj):
        pass

    @property
    def at(self):
        return _At(self)

    # a += b rebinds in JAX; never mutate a shared buffer
    def __iadd__(self, o):
        return self + o

    def __isub__(self, o):
        return self - o

    def __imul__(self, o):
        return self * o

    def __itruediv__(self, o):
        return self / o

    def __ipow__(self, o):
        return self ** o

    def __imatmul__(self, o):
        return self @ o


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIdx(self.arr, idx)


class _AtIdx:
    def __init__(self, arr, idx):
        self.arr = arr
        self.idx = idx

    def _copy(self, value):
        out = np.array(self.arr, copy=True)
        dtype = np.result_type(out.dtype, np.asarray(value).dtype)
        if dtype != out.dtype:
            out = out.astype(dtype)
        return out

    def set(self, value, **_):
        out = self._copy(value)
        out[self.idx] = np.asarray(value)
        return wrap(out)

    def add(self, value, **_):
        out = self._copy(value)
        np.add.at(out, self.idx, np.asarray(value))
        return wrap(out)

    def multiply(self, value, **_):
        out = self._copy(value)
        np.multiply.at(out, self.idx, np.asarray(value))
        return wrap(out)

    def get(self, **_):
        return wrap(np.asarray(self.arr)[self.idx])


def wrap(x):
    if isinstance(x, JArr):
        return x
    if isinstance(x, np.ndarray):
        return x.view(JArr)
    if isinstance(x, (np.generic, float, int, bool, complex)) and not isinstance(x, (str, bytes)):
        return np.asarray(x).view(JArr)
    if isinstance(x, tuple):
        return tuple(wrap(v) for v in x)
    if isinstance(x, list):
        return [wrap(v) for v in x]
    return x


# ----------------------------------------------------------------------------------
# pytrees
# ----------------------------------------------------------------------------------
_REGISTRY: dict = {}


def register(cls, flatten, unflatten):
    _REGISTRY[cls] = (flatten, unflatten)


def _is_leaf(x):
    return x is None or isinstance(x, (np.ndarray, np.generic, float, int, bool, complex))


def flatten(tree):
    """Return (leaves, treedef)."""
    if tree is None:
        return [], ("none",)
    if isinstance(tree, (np.ndarray, np.generic, float, int, bool, complex)):
        return [tree], ("leaf",)
    t = type(tree)
    if t in _REGISTRY:
        children, aux = _REGISTRY[t][0](tree)
        leaves, defs = [], []
        for c in children:
            lv, d = flatten(c)
            leaves += lv
            defs.append((d, len(lv)))
        return leaves, ("reg", t, aux, defs)
    if isinstance(tree, (tuple, list)):
        leaves, defs = [], []
        for c in tree:
            lv, d = flatten(c)
            leaves += lv
            defs.append((d, len(lv)))
        return leaves, ("seq", t, defs)
    if isinstance(tree, dict):
        keys = sorted(tree)
        leaves, defs = [], []
        for k in keys:
            lv, d = flatten(tree[k])
            leaves += lv
            defs.append((d, len(lv)))
        return leaves, ("dict", keys, defs)
    return [tree], ("leaf",)


def unflatten(treedef, leaves):
    leaves = list(leaves)
    kind = treedef[0]
    if kind == "none":
        return None
    if kind == "leaf":
        return leaves[0]

    def rebuild(defs):
        out, i = [], 0
        for d, n in defs:
            out.append(unflatten(d, leaves[i:i + n]))
            i += n
        return out

    if kind == "reg":
        _, t, aux, defs = treedef
        return _REGISTRY[t][1](aux, tuple(rebuild(defs)))
    if kind == "seq":
        _, t, defs = treedef
        vals = rebuild(defs)
        return t(vals) if t is not tuple else tuple(vals)
    if kind == "dict":
        _, keys, defs = treedef
        return dict(zip(keys, rebuild(defs)))
    raise TypeError(treedef)


def tree_map(f, tree, *rest, is_leaf=None):
    leaves, td = flatten(tree)
    others = [flatten(r)[0] for r in rest]
    return unflatten(td, [f(x, *xs) for x, *xs in zip(leaves, *others)])


# ----------------------------------------------------------------------------------
# transformations
# ----------------------------------------------------------------------------------
def _take(tree, axis, i):
    if axis is None:
        return tree
    return tree_map(lambda a: wrap(np.take(np.asarray(a), i, axis=axis)), tree)


def _size(tree, axis):
    leaves, _ = flatten(tree)
    for a in leaves:
        if a is not None:
            return np.shape(a)[axis]
    raise ValueError("vmap over an empty tree")


def _stack(outs, axis):
    leaves0, td = flatten(outs[0])
    cols = [flatten(o)[0] for o in outs]
    stacked = [wrap(np.stack([np.asarray(c[k]) for c in cols], axis=axis)) for k in range(len(leaves0))]
    return unflatten(td, stacked)


def vmap(f, in_axes=0, out_axes=0, **_):
    def wrapped(*args):
        ia = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, ia):
            if ax is not None:
                n = _size(a, ax)
                break
        if n is None:
            raise ValueError("vmap with no mapped axis")
        outs = [f(*[_take(a, ax, i) for a, ax in zip(args, ia)]) for i in range(n)]
        if n == 0:
            raise ValueError("vmap over a zero-length axis")
        oa = out_axes
        if isinstance(outs[0], tuple) and isinstance(oa, (tuple, list)):
            return tuple(_stack([o[k] for o in outs], oa[k]) for k in range(len(oa)))
        return _stack(outs, oa)

    return wrapped


def lax_map(f, xs, batch_size=None):
    n = _size(xs, 0)
    if n == 0:
        raise ValueError("lax.map over a zero-length axis")
    outs = [f(_take(xs, 0, i)) for i in range(n)]
    return _stack(outs, 0)
