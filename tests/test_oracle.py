"""The FP64 oracle against the reference's own known-answer and property tests.

The reference has no stored numeric fixtures; its tests check kernel known answers and
physical properties.  These are ported here against the oracle (CPU only).
"""
from __future__ import annotations

import numpy as np
import pytest

from flapjax_b200 import cases
from oracle import uvlm_ref as R


def test_kernel_known_answers():
    """tests/algebra/test_kernels.py:9-98."""
    y = np.array([[0.0, 1.0, 0.0], [0.0, -1.0, 0.0]])
    assert np.all(np.isnan(R.bs_plain(np.zeros(3), y[0], y[1])))
    assert np.all(np.isnan(R.bs_plain(np.array([0.0, 1.0, 0.0]), np.zeros(3), np.array([0.0, -1.0, 0.0]))))
    x = np.array([0.1, 0.0, 0.0])
    assert not np.all(np.isnan(R.bs_plain(x, y[0], y[1])))
    assert np.allclose(R.bs_epsilon(np.zeros(3), y[0], y[1]), 0.0)
    assert np.allclose(R.bs_epsilon(np.array([0.0, 1.0, 0.0]), np.zeros(3), np.array([0.0, -1.0, 0.0])), 0.0)
    assert np.allclose(R.bs_plain(x, y[0], y[1]), R.bs_epsilon(x, y[0], y[1]), rtol=5e-5)
    assert np.allclose(R.bs_cutoff(np.zeros(3), y[0], y[1]), 0.0)
    assert np.allclose(R.bs_cutoff(np.array([0.0, 1.0, 0.0]), np.zeros(3), np.array([0.0, -1.0, 0.0])), 0.0)
    xo = np.array([1.01 * R.R_CUTOFF, 0.0, 0.0])
    assert np.allclose(R.bs_plain(xo, y[0], y[1]), R.bs_cutoff(xo, y[0], y[1]))
    assert np.allclose(R.bs_cutoff(np.array([0.99 * R.R_CUTOFF, 0.0, 0.0]), y[0], y[1]), 0.0)


def test_kernel_finite_segment_closed_form():
    """Straight filament of half-length L seen from distance h on its bisector:
    |v| = (1 / (4 pi h)) * 2L / sqrt(L^2 + h^2).  The epsilon kernel's regulariser
    EPSILON |r0|^4 scales with the fourth power of the filament length, so it is checked
    on a short filament only."""
    h, L = 0.3, 10.0
    want = 2 * L / np.sqrt(L * L + h * h) / (4 * np.pi * h)
    x = np.array([h, 0.0, 0.0])
    y0, y1 = np.array([0.0, -L, 0.0]), np.array([0.0, L, 0.0])
    assert np.isclose(np.linalg.norm(R.bs_plain(x, y0, y1)), want, rtol=1e-13)
    assert np.isclose(np.linalg.norm(R.bs_epsilon(x, y0, y1)), want, rtol=1e-3)
    assert np.isclose(np.linalg.norm(R.bs_epsilon(x, y0 / 100, y1 / 100)),
                      2 * 0.1 / np.sqrt(0.01 + h * h) / (4 * np.pi * h), rtol=1e-9)


def _square_wing(u_inf):
    mn, width = 5, 1.0
    hg = np.zeros((mn + 1, 4, 4))
    hg[:, :3, :3] = np.eye(3)
    hg[:, 1, 3] = np.linspace(0.0, width, mn + 1)
    uv = R.UVLMRef([(mn, mn, 0)], np.arange(mn + 1))
    uv.set_design_variables(1.0, R.Constant(u_inf, 1.225, True), R.make_rectangular_grid(mn, mn, width, 0.0), hg)
    return uv


def test_rotation_invariance_no_wake():
    """tests/aero/test_static_no_wake.py:11-65."""
    a = _square_wing(np.array((0.0, 10.0, 3.0))).solve_static()
    b = _square_wing(np.array((10.0, 0.0, 3.0))).solve_static()
    assert np.allclose(a.gamma_b[0][0], b.gamma_b[0][0])
    assert np.allclose(np.sum(a.f_steady[0][0]), 0.0, atol=1e-5, rtol=1e-4)
    assert np.allclose(a.f_steady[0][0], np.transpose(b.f_steady[0][0], (1, 0, 2))[..., (1, 0, 2)], atol=1e-5,
                       rtol=1e-4)


def test_mirror_equals_full_wing():
    """tests/aero/test_mirrored_wing.py:11-78."""
    m, n, m_star, c_ref, b_ref = 5, 10, 20, 1.0, 5.0
    u_inf = np.array((10.0, 0.0, 1.0))
    dt = c_ref / (np.linalg.norm(u_inf) * m)
    ff = R.Constant(u_inf, 1.225, True)
    hg = np.zeros((n + 1, 4, 4))
    hg[:, :3, :3] = np.eye(3)
    hg[:, 1, 3] = np.linspace(0.0, b_ref, n + 1)
    um = R.UVLMRef([(m, n, m_star)], np.arange(n + 1), mirror_point=np.zeros(3), mirror_normal=np.array((0.0, 1.0, 0.0)))
    um.set_design_variables(dt, ff, R.make_rectangular_grid(m, n, c_ref, 0.0), hg)
    sm = um.solve_static()
    hg2 = np.zeros((2 * n + 1, 4, 4))
    hg2[:, :3, :3] = np.eye(3)
    hg2[:, 1, 3] = np.linspace(-b_ref, b_ref, 2 * n + 1)
    uf = R.UVLMRef([(m, 2 * n, m_star)], np.arange(2 * n + 1))
    uf.set_design_variables(dt, ff, R.make_rectangular_grid(m, 2 * n, c_ref, 0.0), hg2)
    sf = uf.solve_static()
    assert np.allclose(sm.gamma_b[0][0], sf.gamma_b[0][0][:, n:])
    assert np.allclose(sm.gamma_w[0][0], sf.gamma_w[0][0][:, n:])


def test_static_wake_and_steady_kutta():
    """Static solve: the wake carries the TE circulation on every row (uvlm.py:995-1012)."""
    c = cases.wing_heave(m=4, n=6, m_star=8, n_steps=1)
    uv = R.UVLMRef([(c.m, c.n, c.m_star)], np.arange(c.n + 1))
    uv.set_design_variables(c.dt, R.Constant(c.u_inf, c.rho, True), c.zeta_b0, c.hg0)
    st = uv.solve_static()
    assert np.allclose(st.gamma_w[0][0], st.gamma_b[0][0][-1][None, :])


@pytest.mark.slow
def test_variable_wake_matches_uniform():
    """tests/aero/test_variable_wake_disc.py:12-89 (shortened to 0.5 s of heave)."""
    u_inf = np.array((10.0, 0.0, 0.0))
    m, n, m_star, c_ref, b_ref = 6, 12, 40, 1.0, 5.0
    ff = R.Constant(u_inf, 1.225, True)
    dt = c_ref / (m * ff.u_inf_mag)
    n_tstep = int(np.ceil(0.5 / dt))
    x_grid = R.make_rectangular_grid(m, n, c_ref, 0.0)
    hg = np.zeros((n + 1, 4, 4))
    hg[:, 3, 3] = 1.0
    hg[:, :3, :3] = np.eye(3)
    hg[:, 1, 3] = np.linspace(0.0, b_ref, n + 1)
    omega, ampl = 2 * np.pi * 3.0, 0.1
    t = np.arange(n_tstep) * dt
    hg_t = np.repeat(hg[None], n_tstep, axis=0)
    hg_t[:, :, 2, 3] += (ampl * 0.5 * (1.0 - np.cos(omega * t)))[:, None]
    hg_dot_t = np.zeros_like(hg_t)
    hg_dot_t[:, :, 2, 3] = (ampl * omega * 0.5 * np.sin(omega * t))[:, None]
    out = []
    for dw in (np.ones(m_star) * dt * ff.u_inf_mag, None):
        uv = R.UVLMRef([(m, n, m_star)], np.arange(n + 1), gamma_dot_relaxation=1.0)
        uv.set_design_variables(dt, ff, x_grid, hg, delta_w=dw)
        out.append(uv.solve_prescribed_dynamic(uv.solve_static(), hg_t, hg_dot_t).gamma_b[0])
    assert np.allclose(out[0], out[1], atol=1e-3)


def test_split_and_average_helpers():
    a = np.arange(12.0).reshape(3, 4)
    s = R.split_to_vertex(a, (0, 1))
    assert s.shape == (4, 5)
    assert np.isclose(s.sum(), a.sum())
    assert np.allclose(R.neighbour_average(np.arange(5.0), 0), [0.5, 1.5, 2.5, 3.5])


def test_cpp_oracle_matches_numpy_oracle():
    """The C++/OpenMP restatement of the pair sums (CPU baseline) against the NumPy oracle:
    every kernel, with and without a mirror plane, static AIC with wake lumping, and a
    short free-wake run.  The sums are accumulated in another order (per target over all
    filaments instead of per lattice), hence 1e-10 on the velocities at random points."""
    import subprocess
    from pathlib import Path

    subprocess.run(["make", "-s", "-C", str(Path(__file__).resolve().parents[1] / "oracle")], check=True)
    from flapjax_b200 import cases
    from oracle import uvlm_cpp as CP
    from tests.helpers import rel_err

    rng = np.random.default_rng(0)
    c = cases.wing_free(m=4, n=8, m_star=6, n_steps=4, seed=1)
    zb = c.zeta_b0
    zw = zb[-1][None] + np.arange(7)[:, None, None] * np.array([0.25, 0.0, 0.02])
    gb, gw = rng.normal(size=(4, 8)), rng.normal(size=(6, 8))
    tg = rng.normal(size=(50, 3)) + [0.5, 4.0, 0.0]
    cc, nc = R.compute_surf_c(zb), R.compute_surf_nc(zb)
    for kern, rc in ((R.KERNEL_EPSILON, 1e-4), (R.KERNEL_CUTOFF, 1e-3), (R.KERNEL_PLAIN, 0.0)):
        for mir in (None, (np.array([0.0, -0.5, 0.0]), np.array([0.0, 1.0, 0.0]))):
            assert rel_err(CP.compute_v_ind(tg, [zb, zw], [gb, gw], kern, mir, rc),
                           R.compute_v_ind(tg, [zb, zw], [gb, gw], kern, mir, rc)) < 1e-10
            for wake in (None, [zw]):
                assert rel_err(CP.compute_aic_solve([cc], [nc], [zb], wake, kern, mir, rc),
                               R.compute_aic_solve([cc], [nc], [zb], wake, kern, mir, rc)) < 1e-11

    def run(cls):
        uv = cls([(c.m, c.n, c.m_star)], np.arange(c.n + 1), kernel=c.kernel, r_cut=c.r_cut, free_wake=True)
        uv.set_design_variables(c.dt, R.Constant(c.u_inf, c.rho, True), c.zeta_b0, c.hg0)
        return uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)

    a, b = run(CP.UVLMCpp), run(R.UVLMRef)
    for f in ("gamma_b", "gamma_w", "zeta_w", "f_steady", "f_unsteady"):
        assert rel_err(getattr(a, f)[0], getattr(b, f)[0]) < 1e-12, f
