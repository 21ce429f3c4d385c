"""Background flow fields (mirrors ``flapjax.aero.flowfields``, aero/flowfields.py:13-200).

The flow is evaluated inside the CUDA kernels; these classes carry its parameters to the
library (``to_c``) and evaluate it on the host for callers that need it.
"""
from __future__ import annotations

import numpy as np

from . import _lib


def _vec3(x, name):
    a = np.asarray(x, dtype=np.float64)
    if a.shape != (3,):
        raise ValueError(f"Expected {name} to have shape (3,), got {a.shape}")
    return a


class FlowField:
    """Base flow field, aero/flowfields.py:13-37."""

    def __init__(self, u_inf, rho, relative_motion):
        self.u_inf = _vec3(u_inf, "u_inf")
        self.rho = float(rho)
        self.u_inf_mag = float(np.linalg.norm(self.u_inf))
        if self.u_inf_mag == 0.0:
            raise ValueError("u_inf must be non-zero")
        self.u_inf_dir = self.u_inf / self.u_inf_mag
        self.q_inf = 0.5 * self.rho * self.u_inf_mag**2
        self.relative_motion = bool(relative_motion)

    def __call__(self, x, t):
        raise NotImplementedError

    def vmap_call(self, x, t):
        """Evaluate at coordinates ``(..., 3)`` (aero/flowfields.py:49-60)."""
        return self(np.asarray(x, dtype=np.float64), float(t))

    def to_c(self) -> _lib.FjFlowfield:
        raise NotImplementedError


class Constant(FlowField):
    """Constant velocity field, aero/flowfields.py:87-97."""

    def __call__(self, x, t):
        out = np.zeros(np.shape(x), dtype=np.float64)
        if self.relative_motion:
            out[...] = self.u_inf
        return out

    def to_c(self) -> _lib.FjFlowfield:
        f = _lib.FjFlowfield()
        f.kind = _lib.FJ_FLOW_CONSTANT
        f.relative_motion = int(self.relative_motion)
        f.u_inf[:] = self.u_inf.tolist()
        f.rho = self.rho
        return f


class OneMinusCosine(FlowField):
    """1-cos gust, aero/flowfields.py:100-181: ``0.5 A (1 - cos(pi s / L))`` for
    ``0 < s < 2L``, so ``gust_length`` L is half of the full gust length."""

    def __init__(self, u_inf, rho, relative_motion, gust_length, gust_amplitude, gust_travel_direction=None,
                 gust_amplitude_direction=None, gust_x0=None):
        super().__init__(u_inf, rho, relative_motion)
        self.gust_amplitude = float(gust_amplitude)
        self.gust_length = float(gust_length)
        d = self.u_inf_dir if gust_travel_direction is None else _vec3(gust_travel_direction, "gust_travel_direction")
        self.gust_travel_direction = d / np.linalg.norm(d)
        a = np.array((0.0, 0.0, 1.0)) if gust_amplitude_direction is None else _vec3(
            gust_amplitude_direction, "gust_amplitude")
        self.gust_amplitude_direction = a / np.linalg.norm(a)
        self.gust_x0 = np.zeros(3) if gust_x0 is None else _vec3(gust_x0, "gust_x0")

    def __call__(self, x, t):
        x = np.asarray(x, dtype=np.float64)
        rel_x = x - self.gust_x0
        if self.relative_motion:
            rel_x = rel_x - self.u_inf * t
        gx = rel_x @ self.gust_travel_direction
        val = (self.gust_amplitude_direction * self.gust_amplitude * 0.5
               * (1.0 - np.cos(np.pi * gx[..., None] / self.gust_length)))
        u = np.where(((gx > 0) & (gx < 2.0 * self.gust_length))[..., None], val, 0.0)
        if self.relative_motion:
            u = u + self.u_inf
        return u

    def to_c(self) -> _lib.FjFlowfield:
        f = _lib.FjFlowfield()
        f.kind = _lib.FJ_FLOW_ONE_MINUS_COSINE
        f.relative_motion = int(self.relative_motion)
        f.u_inf[:] = self.u_inf.tolist()
        f.rho = self.rho
        f.gust_length = self.gust_length
        f.gust_amplitude = self.gust_amplitude
        f.gust_travel_dir[:] = self.gust_travel_direction.tolist()
        f.gust_amplitude_dir[:] = self.gust_amplitude_direction.tolist()
        f.gust_x0[:] = self.gust_x0.tolist()
        return f
