import numpy as _np

from ._core import flatten, unflatten, wrap


def ravel_pytree(tree):
    leaves, td = flatten(tree)
    shapes = [_np.shape(x) for x in leaves]
    flat = wrap(_np.concatenate([_np.ravel(x) for x in leaves])) if leaves else wrap(_np.zeros(0))

    def unravel(v):
        out, i = [], 0
        for s in shapes:
            n = int(_np.prod(s))
            out.append(wrap(_np.asarray(v[i:i + n]).reshape(s)))
            i += n
        return unflatten(td, out)

    return flat, unravel
