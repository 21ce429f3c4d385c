"""Vector-Jacobian products of the epsilon Biot-Savart kernel (TEST INFRASTRUCTURE ONLY).

The reference obtains gradients by reverse-mode AD of ``biot_savart_epsilon``
(aero/utils.py:606-623) through ``jax.vjp``.  This is the same derivative written out:
for K(r1, r2) = c * dot / (4 pi D) with r1 = x - y0, r2 = x - y1, r0 = y1 - y0,
c = r1 x r2, u_i = r_i / sqrt(|r_i|^2 + eps^2), dot = r0 . (u1 - u2),
D = |c|^2 + eps |r0|^4, and a cotangent lam:

    d(lam.K)/dr1 = s (r2 x lam) + a [ddot/dr1 / (4 pi D) - dot dD/dr1 / (4 pi D^2)]
    d(lam.K)/dr2 = s (lam x r1) + a [ddot/dr2 / (4 pi D) - dot dD/dr2 / (4 pi D^2)]

with a = lam.c, s = dot / (4 pi D), ddot/dr1 = (u1 - u2) + (r0 - (r0.u1) u1) / n1,
ddot/dr2 = -(u1 - u2) - (r0 - (r0.u2) u2) / n2, dD/dr1 = 2 (r2 x c) + 4 eps |r0|^2 r0,
dD/dr2 = 2 (c x r1) - 4 eps |r0|^2 r0.  Then x_bar = d/dr1 + d/dr2, y0_bar = -d/dr1,
y1_bar = -d/dr2.  The cutoff kernel (aero/utils.py:626-648) is the same with D = |c|^2
(no eps term) and zero -- derivative included -- where the target lies within r_cut of the
filament line.  Used by the tests as the checker of the CUDA adjoint kernels.
"""
from __future__ import annotations

import numpy as np

from .uvlm_ref import EPSILON, KERNEL_CUTOFF, KERNEL_EPSILON, R_CUTOFF


def bs_epsilon_vjp(x, y0, y1, lam):
    """(x_bar, y0_bar, y1_bar) of lam . biot_savart_epsilon(x, (y0, y1)); broadcasting (..., 3)."""
    return bs_vjp(x, y0, y1, lam, KERNEL_EPSILON)


def bs_vjp(x, y0, y1, lam, kernel=KERNEL_EPSILON, r_cut=R_CUTOFF):
    """(x_bar, y0_bar, y1_bar) of lam . K(x, (y0, y1)) for the epsilon or cutoff kernel."""
    with np.errstate(divide="ignore", invalid="ignore"):  # masked cutoff pairs may divide by 0
        return _bs_vjp(x, y0, y1, lam, kernel, r_cut)


def _bs_vjp(x, y0, y1, lam, kernel, r_cut):
    r0 = y1 - y0
    r1 = x - y0
    r2 = x - y1
    n1 = np.sqrt(np.sum(r1 * r1, -1) + EPSILON * EPSILON)[..., None]
    n2 = np.sqrt(np.sum(r2 * r2, -1) + EPSILON * EPSILON)[..., None]
    u1, u2 = r1 / n1, r2 / n2
    c = np.cross(r1, r2)
    dot = np.sum(r0 * (u1 - u2), -1)[..., None]
    r0sq = np.sum(r0 * r0, -1)[..., None]
    eps = EPSILON if kernel == KERNEL_EPSILON else 0.0
    D = np.sum(c * c, -1)[..., None] + eps * r0sq * r0sq
    s = dot / (4 * np.pi * D)
    a = np.sum(lam * c, -1)[..., None]
    ddot1 = (u1 - u2) + (r0 - np.sum(r0 * u1, -1)[..., None] * u1) / n1
    ddot2 = -(u1 - u2) - (r0 - np.sum(r0 * u2, -1)[..., None] * u2) / n2
    dD1 = 2 * np.cross(r2, c) + 4 * eps * r0sq * r0
    dD2 = 2 * np.cross(c, r1) - 4 * eps * r0sq * r0
    g1 = s * np.cross(r2, lam) + a * (ddot1 / (4 * np.pi * D) - dot * dD1 / (4 * np.pi * D * D))
    g2 = s * np.cross(lam, r1) + a * (ddot2 / (4 * np.pi * D) - dot * dD2 / (4 * np.pi * D * D))
    if kernel == KERNEL_CUTOFF:
        sm = np.sum(r0 * r1, -1)[..., None] / r0sq
        keep = np.linalg.norm(r1 - sm * r0, axis=-1)[..., None] > r_cut
        g1 = np.where(keep, g1, 0.0)
        g2 = np.where(keep, g2, 0.0)
    return g1 + g2, -g1, -g2
