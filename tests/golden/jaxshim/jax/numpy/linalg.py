import numpy as _np

from .._core import wrap


def __getattr__(name):
    obj = getattr(_np.linalg, name)
    if callable(obj):
        return lambda *a, **k: wrap(obj(*a, **k))
    return obj
