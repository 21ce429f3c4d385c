"""The time-step residual VJP (flapjax_b200.residual, the VJP the reference takes with
jax.vjp of UVLM.timestep_residual, aero/uvlm.py:1942-2047) with the oracle standing in for
the device, against the restated residual (oracle/uvlm_residual.py): its value, and
<r_bar, J d> from extended-precision central differences against <J^T r_bar, d> for random
directions d in every input (states of n and n-1, node frames and their velocities,
the beam forces).  The restated residual vanishes on the oracle forward's own states."""
from __future__ import annotations

import numpy as np
import pytest

from flapjax_b200 import cases
from flapjax_b200.residual import AeroResidual
from oracle import uvlm_ref as R
from oracle import uvlm_residual as RR
from tests.adjoint_oracle import OracleDev
from tests.helpers import oracle_uvlm

_ST = ("gamma_b", "gamma_w", "gamma_b_dot", "zeta_w")


def _setup(builder, gust=None):
    c = {"heave": lambda: cases.wing_heave(m=3, n=4, m_star=4, n_steps=3),
         "free": lambda: cases.wing_free(m=3, n=4, m_star=4, n_steps=3, seed=1)}[builder]()
    uv, _ = oracle_uvlm(c, gust=gust)
    out = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    n = 2
    q = lambda i: {k: [np.array(a[i]) for a in getattr(out, k)] for k in _ST}
    ft = [fs[n] + fu[n] for fs, fu in zip(out.f_steady, out.f_unsteady)]
    rm = c.hg_t[n][:, :3, :3]
    fb = RR.transform_nodal_vect(RR.project_forcing_to_beam(ft, rm, uv.dof_mapping, uv.zeta_b0),
                                 np.swapaxes(rm, -2, -1))
    return c, uv, out, n, q(n), q(n - 1), fb


@pytest.mark.parametrize("builder", ["heave", "free"])
def test_residual_vanishes_on_forward_states(builder):
    c, uv, out, n, qn, qm, fb = _setup(builder)
    r = RR.timestep_residual(uv, out.t[n], c.hg_t[n], c.hg_dot_t[n], c.hg_t[n - 1], qn, qm, fb)
    assert np.max(np.abs(r)) < 1e-12


@pytest.mark.parametrize("builder,gust", [("heave", None), ("free", None),
                                          ("free", dict(gust_length=2.0, gust_amplitude=0.1,
                                                        gust_x0=np.array([-3.0, 0.0, 0.0])))])
def test_residual_vjp_matches_finite_differences(builder, gust):
    c, uv, out, n, qn, qm, fb = _setup(builder, gust)
    rng = np.random.default_rng(7)
    # move the states off the forward's solution so that every term is exercised
    qn = {k: [a + 0.01 * rng.normal(size=a.shape) for a in v] for k, v in qn.items()}
    fb = fb + 0.01 * rng.normal(size=fb.shape)
    t = out.t[n]
    args = (c.hg_t[n], c.hg_dot_t[n], c.hg_t[n - 1])
    r_want = RR.timestep_residual(uv, t, *args, qn, qm, fb)
    ar = AeroResidual(uv, dev=OracleDev(uv.kernel, uv.r_cut, uv.mirror))
    rbar = rng.normal(size=r_want.shape)
    r_got, cot = ar.vjp(t, *args, qn, qm, fb, rbar)
    assert np.max(np.abs(r_got - r_want)) < 1e-12 * max(1.0, np.max(np.abs(r_want)))
    # one random direction in all inputs at once
    dq_n = {k: [rng.normal(size=a.shape) for a in v] for k, v in qn.items()}
    dq_m = {k: [rng.normal(size=a.shape) for a in v] for k, v in qm.items()}
    dh = [rng.normal(size=a.shape) * 0.1 for a in args]
    for a in dh:
        a[:, 3, :] = 0.0   # the homogeneous row is not an input
    dfb = rng.normal(size=fb.shape)
    ad = sum(np.sum(g * d) for k in _ST for g, d in zip(cot["q_n"][k], dq_n[k]))
    ad += sum(np.sum(g * d) for k in _ST for g, d in zip(cot["q_nm1"][k], dq_m[k]))
    ad += sum(np.sum(cot[k] * d) for k, d in zip(("hg_n", "hg_dot_n", "hg_nm1"), dh))
    ad += np.sum(cot["f_beam_n"] * dfb)

    def res(h):
        L = np.longdouble
        qa = {k: [L(a) + h * d for a, d in zip(qn[k], dq_n[k])] for k in _ST}
        qb = {k: [L(a) + h * d for a, d in zip(qm[k], dq_m[k])] for k in _ST}
        ha = [L(a) + h * d for a, d in zip(args, dh)]
        with R.real_type(np.longdouble):
            u, _ = oracle_uvlm(c, gust=gust)
            return RR.timestep_residual(u, L(t), *ha, qa, qb, L(fb) + h * dfb)

    h = np.longdouble(1e-6)
    fd = float(np.sum(rbar * (res(h) - res(-h))) / (2 * h))
    assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)
