"""The time-step residual VJP on the device (fj_vind / fj_vind_vjp / fj_aic_assemble /
fj_lu_* behind flapjax_b200.residual.AeroResidual) against the same sweep over the oracle
(whose algebra tests/test_residual_cpu.py checks by central differences): the residual
and every cotangent, for prescribed and free wakes, delta_w, a mirror plane and two
surfaces."""
from __future__ import annotations

import numpy as np
import pytest

from flapjax_b200 import cases
from flapjax_b200.residual import AeroResidual
from oracle import uvlm_residual as RR
from tests.adjoint_oracle import OracleDev, two_surface_case, two_surface_oracle
from tests.helpers import device_uvlm, oracle_uvlm

pytestmark = pytest.mark.gpu
_ST = ("gamma_b", "gamma_w", "gamma_b_dot", "zeta_w")


def _states(out, i):
    return {k: [np.array(a[i]) for a in getattr(out, k)] for k in _ST}


def _compare(dev_ar, ref_ar, t, hg, hgd, hg1, qn, qm, fb, rng):
    rbar = rng.normal(size=AeroResidual.ravel(qn).size + fb.size)
    r_o, c_o = ref_ar.vjp(t, hg, hgd, hg1, qn, qm, fb, rbar)
    r_d, c_d = dev_ar.vjp(t, hg, hgd, hg1, qn, qm, fb, rbar)
    assert np.max(np.abs(r_d - r_o)) <= 1e-10 * max(1.0, np.max(np.abs(r_o)))
    flat = lambda cot: np.concatenate([np.concatenate([np.ravel(a) for a in cot["q_n"][k]]) for k in _ST]
                                      + [np.concatenate([np.ravel(a) for a in cot["q_nm1"][k]]) for k in _ST]
                                      + [np.ravel(cot[k]) for k in ("hg_n", "hg_dot_n", "hg_nm1", "f_beam_n")])
    a, b = flat(c_d), flat(c_o)
    assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(b))


@pytest.mark.parametrize("variant", ["heave", "free", "free_delta_w", "mirror"])
def test_device_residual_vjp_matches_oracle(cuda, variant):
    rng = np.random.default_rng(11)
    c = (cases.wing_free(m=3, n=5, m_star=5, n_steps=3, seed=2) if variant.startswith("free")
         else cases.wing_heave(m=3, n=5, m_star=5, n_steps=3))
    kw = {}
    if variant == "mirror":
        kw["mirror"] = (np.zeros(3), np.array([0.0, 1.0, 0.0]))
    dw = c.dt * c.u_mag * 1.2 ** np.arange(c.m_star) if variant == "free_delta_w" else None
    ref, ff = oracle_uvlm(c, **kw)
    if dw is not None:
        ref.set_design_variables(c.dt, ff, c.zeta_b0, c.hg0, delta_w=[dw])
    out = ref.solve_prescribed_dynamic(ref.solve_static(), c.hg_t, c.hg_dot_t)
    uv, uff = device_uvlm(c, "fp64", **kw)
    if dw is not None:
        uv.set_design_variables(dt=c.dt, flowfield=uff, zeta_b0=c.zeta_b0, hg0=c.hg0, delta_w=[dw])
    n = 2
    qn = {k: [a + 0.01 * rng.normal(size=a.shape) for a in v] for k, v in _states(out, n).items()}
    qm = _states(out, n - 1)
    fb = rng.normal(size=(c.hg0.shape[0], 6))
    _compare(AeroResidual(uv, cuda), AeroResidual(ref, dev=OracleDev(ref.kernel, ref.r_cut, ref.mirror)),
             out.t[n], c.hg_t[n], c.hg_dot_t[n], c.hg_t[n - 1], qn, qm, fb, rng)


def test_device_residual_vjp_two_surfaces(cuda):
    import flapjax_b200 as fj

    rng = np.random.default_rng(12)
    surfs, hg0, hg_t, hg_dot_t, wing = two_surface_case(True, n_steps=3)
    ref = two_surface_oracle(surfs, hg0, wing)
    out = ref.solve_prescribed_dynamic(ref.solve_static(), hg_t, hg_dot_t)
    kernel = fj.cutoff_kernel(wing.r_cut) if wing.kernel == "cutoff" else fj.biot_savart_epsilon
    uv = fj.UVLM([fj.GridDiscretisation(m, n, ms) for m, n, ms, _, _ in surfs], [d for *_, d in surfs],
                 kernel=kernel, free_wake=wing.free_wake, precision="fp64")
    uv.set_design_variables(dt=wing.dt, flowfield=fj.Constant(wing.u_inf, wing.rho, True),
                            zeta_b0=[z for *_, z, _ in surfs], hg0=hg0)
    n = 2
    qn = {k: [a + 0.01 * rng.normal(size=a.shape) for a in v] for k, v in _states(out, n).items()}
    fb = rng.normal(size=(hg0.shape[0], 6))
    _compare(AeroResidual(uv, cuda), AeroResidual(ref, dev=OracleDev(ref.kernel, ref.r_cut, ref.mirror)),
             out.t[n], hg_t[n], hg_dot_t[n], hg_t[n - 1], qn, _states(out, n - 1), fb, rng)
