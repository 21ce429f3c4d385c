"""The reference's physics-property tests, run on the CUDA path.

* Pseudo-infinite mirrored wing: the inboard strip angles of attack match the geometric
  angle within 2 % (tests/aero/test_infinite_wing_polar.py:53-68 of the reference).
* A rigid wing started from its static solution and left still stays at that solution
  (the aero counterpart of tests/coupled/dynamic/test_dynamic_equilibrium.py:205-266):
  the static solve's lumped wake is the steady dynamic wake.
* Rotation invariance and zero force without a wake
  (tests/aero/test_static_no_wake.py:11-65).
"""
from __future__ import annotations

import numpy as np
import pytest

import flapjax_b200 as fj
from flapjax_b200 import cases
from tests.helpers import device_uvlm, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pseudo_infinite_wing_strip_alpha(cuda, precision):
    m, n, chord, span, u_mag, ea = 4, 12, 1.0, 48.0, 20.0, 0.25
    alpha = np.deg2rad(3.0)
    u_inf = np.array((u_mag * np.cos(alpha), 0.0, u_mag * np.sin(alpha)))
    hg = np.zeros((n + 1, 4, 4))
    hg[:, :3, :3] = np.eye(3)
    hg[:, 1, 3] = np.linspace(0.0, span, n + 1)
    hg[:, 3, 3] = 1.0
    uv = fj.UVLM([fj.GridDiscretisation(m, n, 2)], np.arange(n + 1), mirror_point=np.zeros(3),
                 mirror_normal=np.array((0.0, 1.0, 0.0)), precision=precision)
    uv.set_design_variables(dt=chord / (u_mag * m), flowfield=fj.Constant(u_inf, 1.225, True),
                            zeta_b0=fj.make_rectangular_grid(m, n, chord, ea), hg0=hg)
    a = uv.solve_static(horseshoe=True).alpha[0]
    interior = a[1:a.shape[0] // 4]
    assert np.max(np.abs(interior - alpha) / alpha) < 0.02


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 1e-6)])
def test_still_wing_stays_at_static_solution(cuda, precision, tol):
    c = cases.wing_heave(m=6, n=16, m_star=30, n_steps=25)
    still = np.repeat(c.hg0[None], c.n_tstep, axis=0)
    uv, _ = device_uvlm(c, precision)
    st = uv.solve_static()
    out = uv.solve_prescribed_dynamic(st, still, np.zeros_like(still))
    for i in range(1, c.n_tstep):
        assert rel_err(out.gamma_b[0][i], st.gamma_b[0]) < tol, i
        assert rel_err(out.gamma_w[0][i], st.gamma_w[0]) < tol, i
    assert np.max(np.abs(out.gamma_b_dot[0])) < tol * np.max(np.abs(st.gamma_b[0])) / c.dt


def test_rotation_invariance_and_no_wake_force(cuda):
    """5 x 5 lattice without a wake: Gamma under flow along x equals Gamma of the
    lattice rotated by 90 deg under flow along y; the total force vanishes."""
    m = n = 5
    z = fj.make_rectangular_grid(m, n, 1.0, 0.25)
    z[..., 1] = np.linspace(0.0, 1.0, n + 1)[None, :]
    hg = np.zeros((n + 1, 4, 4))
    hg[:, :3, :3] = np.eye(3)
    hg[:, 3, 3] = 1.0
    out = []
    for rot in (False, True):
        zz = z.copy()
        u = np.array((1.0, 0.0, 0.1))
        if rot:  # rotate the lattice and the flow by 90 deg about z
            zz[..., 0], zz[..., 1] = -z[..., 1], z[..., 0]
            u = np.array((0.0, 1.0, 0.1))
        uv = fj.UVLM([fj.GridDiscretisation(m, n, 0)], np.arange(n + 1))
        uv.set_design_variables(dt=0.1, flowfield=fj.Constant(u, 1.225, True), zeta_b0=zz, hg0=hg)
        s = uv.solve_static()
        out.append(s)
        ft = s.f_steady[0].reshape(-1, 3).sum(0)
        scale = np.abs(s.f_steady[0]).sum()
        assert np.max(np.abs(ft)) < 1e-10 * scale
    assert rel_err(out[1].gamma_b[0], out[0].gamma_b[0]) < 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nonfinite_inputs_return_an_error_status(cuda, precision):
    """Malformed data injected on the host: a NaN in the lattice makes the static solve
    return FJ_ERR_NONFINITE; a NaN node frame at slot 3 makes the dynamic solve name slot
    3.  The device stays usable afterwards."""
    from flapjax_b200._lib import FJ_ERR_NONFINITE, FjError

    c = cases.wing_heave(m=4, n=8, m_star=8, n_steps=6)
    bad = c.zeta_b0.copy()
    bad[2, 3, 2] = np.nan
    uv = fj.UVLM([fj.GridDiscretisation(c.m, c.n, c.m_star)], np.arange(c.n + 1), precision=precision)
    uv.set_design_variables(dt=c.dt, flowfield=fj.Constant(c.u_inf, c.rho, True), zeta_b0=bad, hg0=c.hg0)
    with pytest.raises(FjError) as e:
        uv.solve_static()
    assert e.value.code == FJ_ERR_NONFINITE
    uv, _ = device_uvlm(c, precision)
    hg = c.hg_t.copy()
    hg[3, 0, 2, 3] = np.nan
    with pytest.raises(FjError) as e:
        uv.solve_prescribed_dynamic(uv.solve_static(), hg, c.hg_dot_t)
    assert e.value.code == FJ_ERR_NONFINITE and "slot 3" in str(e.value)
    good = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    assert np.all(np.isfinite(good.gamma_b[0]))
