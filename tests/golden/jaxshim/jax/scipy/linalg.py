import numpy as _np
import scipy.linalg as _sl

from .._core import wrap


def __getattr__(name):
    obj = getattr(_sl, name)
    if callable(obj):
        return lambda *a, **k: wrap(obj(*a, **k))
    return obj
