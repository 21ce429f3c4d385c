"""The adjoint's algebra on the CPU: the Biot-Savart VJP, the reverse sweep of
``PrescribedAdjoint`` (run over oracle stand-ins for the device calls) and the twist
Jacobian, each against central finite differences (h = 1e-6).

The sweep is checked against differences of the oracle forward evaluated in 80-bit
extended precision: agreement 1e-6 relative.  (In float64 the forward's own roundoff
noise, ~1e-11 relative, limits a central difference at h = 1e-6 to ~1e-4.)"""
from __future__ import annotations

import numpy as np
import pytest

from flapjax_b200 import cases
from flapjax_b200.adjoint import twist_jacobian
from oracle import uvlm_ref as R
from oracle.uvlm_vjp import bs_epsilon_vjp
from tests.adjoint_oracle import OracleAdjoint, central_difference, coefficient_weights, forward_objective
from tests.helpers import oracle_uvlm


def test_bs_epsilon_vjp_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(64, 3))
    y0 = rng.normal(size=(64, 3))
    y1 = y0 + rng.normal(size=(64, 3))
    lam = rng.normal(size=(64, 3))
    xb, y0b, y1b = bs_epsilon_vjp(x, y0, y1, lam)
    h = 1e-6
    for arg, bar in ((0, xb), (1, y0b), (2, y1b)):
        for k in range(3):
            args_p = [x.copy(), y0.copy(), y1.copy()]
            args_m = [x.copy(), y0.copy(), y1.copy()]
            args_p[arg][:, k] += h
            args_m[arg][:, k] -= h
            fd = np.sum(lam * (R.bs_epsilon(*args_p) - R.bs_epsilon(*args_m)), axis=-1) / (2 * h)
            assert np.max(np.abs(fd - bar[:, k])) <= 1e-7 * max(1.0, np.max(np.abs(bar[:, k])))


def test_extended_precision_forward_matches_float64():
    c = cases.wing_pitch(m=3, n=4, m_star=4, n_steps=3, n_ctrl=3, seed=3)
    fw = coefficient_weights(c, "CL")
    j64 = forward_objective(c, c.zeta_b0, fw)
    with R.real_type(np.longdouble):
        jld = forward_objective(c, np.asarray(c.zeta_b0, np.longdouble), fw)
    assert jld.dtype == np.longdouble
    assert abs(float(jld) - j64) < 1e-12 * abs(j64)


@pytest.mark.parametrize("which", ["CL", "CD"])
def test_reverse_sweep_matches_finite_differences(which):
    c = cases.wing_pitch(m=3, n=4, m_star=4, n_steps=5, n_ctrl=3, seed=3)
    fw = coefficient_weights(c, which)
    uv, _ = oracle_uvlm(c)
    J, g = OracleAdjoint(uv).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    assert abs(J - forward_objective(c, c.zeta_b0, fw)) < 1e-13 * max(1.0, abs(J))
    rng = np.random.default_rng(1)
    for _ in range(2):
        d = rng.normal(size=c.zeta_b0.shape) * 0.1
        fd = central_difference(c, d, fw)
        assert abs(fd - np.sum(g * d)) <= 1e-6 * abs(fd), (fd, np.sum(g * d))


def test_checkpoint_interval_does_not_change_the_gradient():
    c = cases.wing_heave(m=3, n=4, m_star=3, n_steps=6)
    fw = coefficient_weights(c, "CL")
    uv, _ = oracle_uvlm(c)
    g = [OracleAdjoint(uv).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=k)[1] for k in (1, 4, 100)]
    assert np.max(np.abs(g[0] - g[1])) < 1e-13 * np.max(np.abs(g[2]))
    assert np.max(np.abs(g[0] - g[2])) < 1e-13 * np.max(np.abs(g[2]))


def test_twist_jacobian_finite_differences():
    m, n, span = 4, 8, 8.0
    ctrl_y = np.linspace(0.0, span, 4)
    span_y = np.linspace(0.0, span, n + 1)
    theta = np.deg2rad(np.array([1.0, -0.5, 2.0, 0.3]))
    jac = twist_jacobian(m, n, 1.0, 0.25, ctrl_y, span_y, np.interp(span_y, ctrl_y, theta), camber=0.03)
    h = 1e-6
    for k in range(len(theta)):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (cases.twisted_grid(m, n, 1.0, 0.25, np.interp(span_y, ctrl_y, tp), 0.03)
              - cases.twisted_grid(m, n, 1.0, 0.25, np.interp(span_y, ctrl_y, tm), 0.03)) / (2 * h)
        assert np.max(np.abs(fd - jac[k])) < 1e-9


def test_reverse_sweep_variable_wake_matches_finite_differences():
    """delta_w: the transpose of the arc-length re-discretisation (through the arc lengths,
    as the reference differentiates it by default) against extended-precision central
    differences."""
    c = cases.wing_pitch(m=3, n=4, m_star=5, n_steps=5, n_ctrl=3, seed=3)
    dw = c.dt * c.u_mag * 1.2 ** np.arange(c.m_star)
    fw = coefficient_weights(c, "CL")
    uv, ff = oracle_uvlm(c)
    uv.set_design_variables(c.dt, ff, c.zeta_b0, c.hg0, delta_w=dw)
    J, g = OracleAdjoint(uv).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    assert abs(J - forward_objective(c, c.zeta_b0, fw, dw)) < 1e-13 * abs(J)
    rng = np.random.default_rng(1)
    for _ in range(2):
        d = rng.normal(size=c.zeta_b0.shape) * 0.1
        fd = central_difference(c, d, fw, delta_w=dw)
        assert abs(fd - np.sum(g * d)) <= 1e-6 * abs(fd), (fd, np.sum(g * d))


@pytest.mark.parametrize("kernel,dw_growth", [("cutoff", None), ("epsilon", None), ("cutoff", 1.15)])
def test_reverse_sweep_free_wake_matches_finite_differences(kernel, dw_growth):
    """Free wake (the convection velocity's VJP, whose bound-lattice share is carried to
    the previous step), with the epsilon or the cutoff kernel and optionally delta_w,
    against extended-precision central differences."""
    c = cases.wing_free(m=3, n=4, m_star=4, n_steps=4, seed=1)
    c = cases.WingCase(**{**c.__dict__, "kernel": kernel, "r_cut": 1e-3 if kernel == "cutoff" else 1e-4})
    dw = None if dw_growth is None else c.dt * c.u_mag * dw_growth ** np.arange(c.m_star)
    fw = coefficient_weights(c, "CL")
    uv, ff = oracle_uvlm(c)
    if dw is not None:
        uv.set_design_variables(c.dt, ff, c.zeta_b0, c.hg0, delta_w=dw)
    J, g = OracleAdjoint(uv).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    assert abs(J - forward_objective(c, c.zeta_b0, fw, dw)) < 1e-13 * abs(J)
    rng = np.random.default_rng(1)
    for _ in range(2):
        d = rng.normal(size=c.zeta_b0.shape) * 0.1
        fd = central_difference(c, d, fw, delta_w=dw)
        assert abs(fd - np.sum(g * d)) <= 1e-6 * abs(fd), (fd, np.sum(g * d))


def test_cutoff_vjp_finite_differences():
    from oracle.uvlm_vjp import bs_vjp

    rng = np.random.default_rng(4)
    x = rng.normal(size=(64, 3))
    y0 = rng.normal(size=(64, 3))
    y1 = y0 + rng.normal(size=(64, 3))
    lam = rng.normal(size=(64, 3))
    xb, y0b, y1b = bs_vjp(x, y0, y1, lam, R.KERNEL_CUTOFF, 1e-3)
    h = 1e-6
    for arg, bar in ((0, xb), (1, y0b), (2, y1b)):
        for k in range(3):
            p, m = [x.copy(), y0.copy(), y1.copy()], [x.copy(), y0.copy(), y1.copy()]
            p[arg][:, k] += h
            m[arg][:, k] -= h
            fd = np.sum(lam * (R.bs_cutoff(*p, 1e-3) - R.bs_cutoff(*m, 1e-3)), axis=-1) / (2 * h)
            assert np.max(np.abs(fd - bar[:, k])) <= 1e-7 * max(1.0, np.max(np.abs(bar[:, k])))


@pytest.mark.parametrize("builder", ["pitch", "free"])
def test_reverse_sweep_mirror_matches_finite_differences(builder):
    """A mirrored half-wing (image lattice across y = 0): the image's VJP reflected back
    onto the original vertices, against extended-precision central differences."""
    mir = (np.zeros(3), np.array([0.0, 1.0, 0.0]))
    c = (cases.wing_pitch(m=3, n=4, m_star=4, n_steps=4, n_ctrl=3, seed=3) if builder == "pitch"
         else cases.wing_free(m=3, n=4, m_star=4, n_steps=3, seed=1))
    fw = coefficient_weights(c, "CL")

    def fwd(z):
        u, _ = oracle_uvlm(cases.WingCase(**{**c.__dict__, "zeta_b0": z}), mirror=mir)
        out = u.solve_prescribed_dynamic(u.solve_static(), c.hg_t, c.hg_dot_t)
        ft = sum(fs.sum(axis=(1, 2)) + fu.sum(axis=(1, 2)) for fs, fu in zip(out.f_steady, out.f_unsteady))
        return np.sum(fw[1:] * ft[1:])

    uv, _ = oracle_uvlm(c, mirror=mir)
    J, g = OracleAdjoint(uv).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    assert abs(J - fwd(c.zeta_b0)) < 1e-13 * abs(J)
    d = np.random.default_rng(1).normal(size=c.zeta_b0.shape) * 0.1
    z, h = np.asarray(c.zeta_b0, np.longdouble), np.longdouble(1e-6)
    with R.real_type(np.longdouble):
        fd = float((fwd(z + h * d) - fwd(z - h * d)) / (2 * h))
    assert abs(fd - np.sum(g * d)) <= 1e-6 * abs(fd)


GUST = dict(gust_length=2.0, gust_amplitude=0.1, gust_x0=np.array([-3.0, 0.0, 0.0]))


@pytest.mark.parametrize("builder", ["pitch", "free"])
def test_reverse_sweep_gust_matches_finite_differences(builder):
    """A 1-cos gust (aero/flowfields.py:100-181) sweeping over the wing: the flow's own
    x-derivative at the collocation points, the filament midpoints and the convected wake
    vertices, against extended-precision central differences."""
    c = (cases.wing_pitch(m=3, n=4, m_star=4, n_steps=4, n_ctrl=3, seed=3) if builder == "pitch"
         else cases.wing_free(m=3, n=4, m_star=4, n_steps=3, seed=1))
    fw = coefficient_weights(c, "CL")

    def fwd(z):
        u, _ = oracle_uvlm(cases.WingCase(**{**c.__dict__, "zeta_b0": z}), gust=GUST)
        out = u.solve_prescribed_dynamic(u.solve_static(), c.hg_t, c.hg_dot_t)
        ft = sum(fs.sum(axis=(1, 2)) + fu.sum(axis=(1, 2)) for fs, fu in zip(out.f_steady, out.f_unsteady))
        return np.sum(fw[1:] * ft[1:])

    uv, _ = oracle_uvlm(c, gust=GUST)
    J, g = OracleAdjoint(uv).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    assert abs(J - fwd(c.zeta_b0)) < 1e-13 * abs(J)
    d = np.random.default_rng(2).normal(size=c.zeta_b0.shape) * 0.1
    z, h = np.asarray(c.zeta_b0, np.longdouble), np.longdouble(1e-6)
    with R.real_type(np.longdouble):
        fd = float((fwd(z + h * d) - fwd(z - h * d)) / (2 * h))
    assert abs(fd - np.sum(g * d)) <= 1e-6 * abs(fd)


@pytest.mark.parametrize("free_wake", [False, True])
def test_reverse_sweep_two_surfaces_matches_finite_differences(free_wake):
    """A wing and a tail: forces, the coupled AIC (one transpose solve over both), each
    surface's wake, and (free wake) every wake convected by all four lattices."""
    from tests.adjoint_oracle import two_surface_case, two_surface_oracle

    surfs, hg0, hg_t, hg_dot_t, wing = two_surface_case(free_wake)
    fw = coefficient_weights(wing, "CL")

    def fwd(zs):
        u = two_surface_oracle(surfs, hg0, wing, zs)
        out = u.solve_prescribed_dynamic(u.solve_static(), hg_t, hg_dot_t)
        ft = sum(fs.sum(axis=(1, 2)) + fu.sum(axis=(1, 2)) for fs, fu in zip(out.f_steady, out.f_unsteady))
        return np.sum(fw[1:] * ft[1:])

    uv = two_surface_oracle(surfs, hg0, wing)
    J, g = OracleAdjoint(uv).gradient(hg_t, hg_dot_t, fw, checkpoint=2)
    z0 = [z for *_, z, _ in surfs]
    assert isinstance(g, list) and len(g) == 2
    assert abs(J - fwd(z0)) < 1e-13 * abs(J)
    rng = np.random.default_rng(4)
    ds = [rng.normal(size=z.shape) * 0.1 for z in z0]
    h = np.longdouble(1e-6)
    with R.real_type(np.longdouble):
        zp = [np.asarray(z, np.longdouble) + h * d for z, d in zip(z0, ds)]
        zm = [np.asarray(z, np.longdouble) - h * d for z, d in zip(z0, ds)]
        fd = float((fwd(zp) - fwd(zm)) / (2 * h))
    ad = sum(float(np.sum(a * d)) for a, d in zip(g, ds))
    assert abs(fd - ad) <= 1e-6 * abs(fd)
    # the tail's own share is not negligible
    assert np.max(np.abs(g[1])) > 1e-3 * np.max(np.abs(g[0]))
