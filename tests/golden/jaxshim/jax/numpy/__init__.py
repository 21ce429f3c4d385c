"""jax.numpy stand-in: NumPy functions returning JArr (float64)."""
from __future__ import annotations

import numpy as _np

from .._core import JArr, wrap
from . import linalg  # noqa: F401

pi = _np.pi
inf = _np.inf
nan = _np.nan
float64 = _np.float64
float32 = _np.float32
int32 = _np.int32
int64 = _np.int64
floating = _np.floating
integer = _np.integer
bool_ = _np.bool_
ndarray = _np.ndarray
newaxis = None


def array(x, dtype=None, copy=True):
    return wrap(_np.array(x, dtype=dtype))


def asarray(x, dtype=None):
    return wrap(_np.array(x, dtype=dtype))


def empty(shape, dtype=None):
    return wrap(_np.zeros(shape, dtype=dtype if dtype is not None else _np.float64))


def empty_like(a, dtype=None):
    return wrap(_np.zeros_like(a, dtype=dtype))


def broadcast_to(a, shape):
    return wrap(_np.array(_np.broadcast_to(a, shape)))


def bincount(x, weights=None, minlength=0, *, length=None):
    n = length if length is not None else minlength
    out = _np.bincount(_np.asarray(x).ravel(), weights=weights, minlength=n)
    return wrap(out[:length] if length is not None else out)


acos = _np.arccos
asin = _np.arcsin
atan = _np.arctan
atan2 = _np.arctan2


def __getattr__(name):
    obj = getattr(_np, name)
    if callable(obj) and not isinstance(obj, type):
        def f(*a, **k):
            return wrap(obj(*a, **k))

        f.__name__ = name
        return f
    return obj


for _n in ("acos", "asin", "atan", "atan2"):
    _f = globals()[_n]
    globals()[_n] = (lambda g: (lambda *a, **k: wrap(g(*a, **k))))(_f)
