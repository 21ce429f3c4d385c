"""jax.lax stand-in (eager control flow)."""
import numpy as _np

from ._core import lax_map, wrap


def rsqrt(x):
    return wrap(1.0 / _np.sqrt(x))


def select(pred, on_true, on_false):
    return wrap(_np.where(pred, on_true, on_false))


def cond(pred, true_fun, false_fun, *operands):
    return true_fun(*operands) if bool(pred) else false_fun(*operands)


def fori_loop(lower, upper, body, init_val, **_):
    v = init_val
    for i in range(int(lower), int(upper)):
        v = body(i, v)
    return v


def while_loop(cond_fun, body_fun, init_val):
    v = init_val
    while bool(cond_fun(v)):
        v = body_fun(v)
    return v


def stop_gradient(x):
    return x


map = lax_map  # noqa: A001
