"""Strip polars for the polar correction (``apply_polar_correction``, aero/utils.py:276-397).

The reference takes any ``alpha -> (cl, cd, cm)`` callable per strip (``PolarFunction``,
aero/utils.py:20).  The correction runs inside the CUDA step, so a polar reaches the device
as a table: ``TabulatedPolar`` holds one (alpha ascending; linear interpolation with the end
values held outside, ``np.interp``), and ``tabulate`` samples any other callable onto one.
A polar that is linear in alpha over the table's range is represented exactly.
"""
from __future__ import annotations

import numpy as np

#: alpha grid used for callables that are not already tables (rad, 0.25 deg apart)
DEFAULT_ALPHA = np.linspace(-np.pi / 2, np.pi / 2, 721)


class TabulatedPolar:
    """alpha (n,) ascending -> (cl, cd, cm) by linear interpolation of the (n,) tables."""

    def __init__(self, alpha, cl, cd, cm):
        self.alpha = np.asarray(alpha, dtype=np.float64).ravel()
        self.cl, self.cd, self.cm = (np.broadcast_to(np.asarray(v, dtype=np.float64).ravel(), self.alpha.shape).copy()
                                     for v in (cl, cd, cm))
        if self.alpha.size < 1:
            raise ValueError("a polar table needs at least one point")
        if np.any(np.diff(self.alpha) < 0):
            raise ValueError("polar alpha must be ascending")

    def __call__(self, a):
        a = np.asarray(a, dtype=np.float64)
        return tuple(np.interp(a, self.alpha, v) for v in (self.cl, self.cd, self.cm))

    def rows(self) -> np.ndarray:
        """(n, 4) table of (alpha, cl, cd, cm)."""
        return np.stack([self.alpha, self.cl, self.cd, self.cm], axis=1)


def tabulate(fn, alpha=None) -> TabulatedPolar:
    """``fn`` as a table over ``alpha`` (default ``DEFAULT_ALPHA``); tables pass through."""
    if isinstance(fn, TabulatedPolar):
        return fn
    alpha = DEFAULT_ALPHA if alpha is None else np.asarray(alpha, dtype=np.float64)
    vals = [fn(float(a)) for a in alpha]
    return TabulatedPolar(alpha, *(np.array([float(v[q]) for v in vals]) for q in range(3)))


def pack_surface(polars, n) -> tuple[int, np.ndarray]:
    """The device block of one surface: n strips x P points x (alpha, cl, cd, cm), P the
    longest table (shorter ones repeat their last row, which interpolation never reads
    inside the table and holds outside it)."""
    if len(polars) != n:
        raise ValueError(f"Expected {n} polar callables, got {len(polars)}")
    tabs = [tabulate(p).rows() for p in polars]
    P = max(t.shape[0] for t in tabs)
    out = np.empty((n, P, 4))
    for j, t in enumerate(tabs):
        out[j, :t.shape[0]] = t
        out[j, t.shape[0]:] = t[-1]
    return P, out
