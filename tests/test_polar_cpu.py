"""Polar correction (aero/utils.py:276-397, uvlm.py:1055-1075) in the oracle, pinned by the
reference's own tests on a pseudo-infinite mirrored wing (tests/aero/test_infinite_wing_polar.py:
73-170): a lift-only polar of half the 2 pi slope, a drag-only polar, and the circulation
scaling, each within 1e-6."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import uvlm_ref as R


def pseudo_infinite_wing(alpha_deg, polars=None, m=4, n=12, chord=1.0, span=48.0, u_mag=20.0, ea=0.25,
                         polar_circulation_scale=0.0):
    """The reference test's wing (tests/aero/test_infinite_wing_polar.py:10-48)."""
    a = np.deg2rad(alpha_deg)
    ff = R.Constant(np.array((u_mag * np.cos(a), 0.0, u_mag * np.sin(a))), 1.225, True)
    hg = np.zeros((n + 1, 4, 4))
    hg[:, :3, :3] = np.eye(3)
    hg[:, 1, 3] = np.linspace(0.0, span, n + 1)
    hg[:, 3, 3] = 1.0
    uv = R.UVLMRef([(m, n, 2)], np.arange(n + 1), mirror_point=np.zeros(3), mirror_normal=np.array((0.0, 1.0, 0.0)),
                   polars=polars, polar_circulation_scale=polar_circulation_scale)
    uv.set_design_variables(chord / (u_mag * m), ff, R.make_rectangular_grid(m, n, chord, ea), hg)
    return uv, a, chord, span, ff


def test_lift_only_polar():
    n = 12
    uv, a, chord, span, ff = pseudo_infinite_wing(3.0, [[lambda x: (np.pi * x, 0.0, 0.0)] * n])
    sol = uv.solve_static(horseshoe=True)
    lift = np.sum(sol.f_steady[0][0] * np.array((-np.sin(a), 0.0, np.cos(a))))
    want = ff.q_inf * chord * (span / n) * np.pi * np.sum(sol.alpha[0][0])
    assert abs(lift - want) < 1e-6 * abs(want)


def test_circulation_scaling():
    n = 12
    ref, *_ = pseudo_infinite_wing(3.0)
    corr, *_ = pseudo_infinite_wing(3.0, [[lambda x: (np.pi * x, 0.0, 0.0)] * n], polar_circulation_scale=1.0)
    s0, s1 = ref.solve_static(horseshoe=True), corr.solve_static(horseshoe=True)
    assert np.max(np.abs(s1.gamma_b[0][0] / s0.gamma_b[0][0] - 0.5)) < 1e-6
    assert np.max(np.abs(s1.gamma_w[0][0] / s0.gamma_w[0][0] - 0.5)) < 1e-6


def test_drag_only_polar():
    n, cd0 = 12, 0.02
    uv, a, chord, span, ff = pseudo_infinite_wing(3.0, [[lambda x: (0.0, cd0, 0.0)] * n])
    sol = uv.solve_static(horseshoe=True)
    drag = np.sum(sol.f_steady[0][0] * np.array((np.cos(a), 0.0, np.sin(a))))
    want = ff.q_inf * chord * (span / n) * cd0 * n
    assert abs(drag - want) < 1e-6 * abs(want)


def test_moment_only_polar_is_a_pure_couple():
    """cm alone: the leading/trailing-edge forces cancel (no net force) and the couple
    about the strip is q c b cm."""
    n, cm0 = 12, -0.05
    uv, a, chord, span, ff = pseudo_infinite_wing(3.0, [[lambda x: (0.0, 0.0, cm0)] * n])
    sol = uv.solve_static(horseshoe=True)
    f = sol.f_steady[0][0]
    assert np.max(np.abs(f.sum(axis=(0, 1)))) < 1e-9 * ff.q_inf * chord * span
    # the couple of strip j: e_n-directed forces at LE (+) and TE (-), one chord apart
    le, te = f[0].sum(axis=0), f[-1].sum(axis=0)
    assert np.allclose(le, -te)
    assert abs(np.linalg.norm(le) - ff.q_inf * chord * (span / n) * abs(cm0) * n) < 1e-9 * np.linalg.norm(le)


def test_tabulated_polar_interpolates_like_np_interp():
    pol = R.TabulatedPolar([-0.1, 0.0, 0.2], [-0.5, 0.0, 1.0], [0.01, 0.0, 0.03], [0.0, -0.1, 0.1])
    assert pol(0.1) == pytest.approx((0.5, 0.015, 0.0))
    assert pol(1.0) == pytest.approx((1.0, 0.03, 0.1))   # held at the end
    assert pol(-1.0) == pytest.approx((-0.5, 0.01, 0.0))
