from fractions import Fraction

import numpy as _np

from .._core import wrap


def bernoulli(n):
    """Bernoulli numbers B_0..B_n (B_1 = -1/2), Akiyama-Tanigawa algorithm."""
    n = int(n)
    out = []
    for m in range(n + 1):
        a = [Fraction(0)] * (m + 1)
        for j in range(m + 1):
            a[j] = Fraction(1, j + 1)
            for k in range(j, 0, -1):
                a[k - 1] = k * (a[k - 1] - a[k])
        out.append(float(a[0]))
    if n >= 1:
        out[1] = -0.5
    return wrap(_np.array(out))
