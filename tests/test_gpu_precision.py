"""The mixed path's force coefficients against the plain FP64 path at full workload size.

The mixed path (FP32 Biot-Savart sums with FP64 accumulation, FP32 factors with FP64
refinement) is held to 1e-6 relative in CL and to 1e-6 of max|CD| in CD:

* 8 x 32 heave, W = 64, 50 steps, and the 12 x 64 pitch + twist wing, W = 100, 1000 steps
  (prescribed wakes): over the whole trajectory (CD can change sign in pitch, so its error
  is taken against max|CD|);
* 16 x 128 free wake, W = 200, cutoff 1e-3: the free wake is chaotic (a 1e-13 change of
  the FP64 input moves its CL by ~1e-4 within 200 steps), so the claim is the one-step
  error: the FP64 state of slot i-1 in, one mixed step, compared with the FP64 step, at
  five slots of a 60-step run.
"""
from __future__ import annotations

import numpy as np
import pytest

from flapjax_b200 import cases

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _device_case(case, precision, n_slots):
    import flapjax_b200 as fj

    kernel = fj.cutoff_kernel(case.r_cut) if case.kernel == "cutoff" else fj.biot_savart_epsilon
    uv = fj.UVLM([fj.GridDiscretisation(case.m, case.n, case.m_star)], np.arange(case.n + 1), kernel=kernel,
                 free_wake=case.free_wake, precision=precision)
    uv.set_design_variables(dt=case.dt, flowfield=fj.Constant(case.u_inf, case.rho, True), zeta_b0=case.zeta_b0,
                            hg0=case.hg0)
    dc = uv.make_device_case(n_slots)
    uv.load_initial(dc, uv.solve_static())
    dc.set_hg(case.hg_t[:n_slots], case.hg_dot_t[:n_slots])
    return dc


def _coeffs(ft, case):
    a = np.deg2rad(case.alpha_deg)
    q = 0.5 * case.rho * case.u_mag ** 2 * case.s_ref
    return ft @ np.array((-np.sin(a), 0.0, np.cos(a))) / q, ft @ np.array((np.cos(a), 0.0, np.sin(a))) / q


@pytest.mark.parametrize("name", ["heave_8x32", "pitch_twist_12x64"])
def test_mixed_trajectory_cl_cd(cuda, name):
    case = cases.wing_heave() if name == "heave_8x32" else cases.wing_pitch(n_steps=1000)
    n = case.n_tstep
    out = {}
    for prec in ("fp64", "mixed"):
        dc = _device_case(case, prec, n)
        dc.solve_dynamic(1, n)
        out[prec] = _coeffs(dc.force_total[1:].cpu().numpy(), case)
        del dc
    (cl64, cd64), (clm, cdm) = out["fp64"], out["mixed"]
    cl_err = float(np.max(np.abs(clm - cl64) / np.abs(cl64)))
    cd_err = float(np.max(np.abs(cdm - cd64)) / np.max(np.abs(cd64)))
    assert cl_err < TOL, cl_err
    assert cd_err < TOL, cd_err


def test_mixed_one_step_cl_cd_free_wake(cuda):
    case = cases.wing_free(n_steps=60)
    n = case.n_tstep
    d64 = _device_case(case, "fp64", n)
    d64.solve_dynamic(1, n)
    dm = _device_case(case, "mixed", n)
    dm.solve_dynamic(1, 2)  # the first (factorising) step
    cl64, cd64 = _coeffs(d64.force_total.cpu().numpy(), case)
    errs = []
    for i in np.linspace(2, n - 1, 5).astype(int):
        dm.copy_slot_from(d64, i - 1)
        dm.solve_dynamic(i, i + 1, reuse_factors=True)
        cl_i, cd_i = _coeffs(dm.force_total[i].cpu().numpy(), case)
        errs.append((abs(cl_i - cl64[i]) / abs(cl64[i]), abs(cd_i - cd64[i]) / np.max(np.abs(cd64[1:]))))
    assert max(e[0] for e in errs) < TOL, errs
    assert max(e[1] for e in errs) < TOL, errs


def test_fp64_reuses_factors_only_for_an_unchanged_lattice(cuda):
    """The FP64 path factors the AIC only when the lattice differs from that of its cached
    factors: a static wing (free wake) after the first step, and a pitching wing every
    step.  Both must equal the oracle-checked direct path: a graph-free run where every
    step is the first of its call (and so always factors)."""
    import torch

    for case in (cases.wing_free(m=4, n=10, m_star=12, n_steps=8), cases.wing_pitch(m=4, n=8, m_star=10, n_steps=8,
                                                                                  n_ctrl=5)):
        n = case.n_tstep
        a = _device_case(case, "fp64", n)
        a.solve_dynamic(1, n)
        b = _device_case(case, "fp64", n)
        for i in range(1, n):
            b.solve_dynamic(i, i + 1)
        torch.cuda.synchronize()
        ga, gb = a.arrays["gamma_b"].cpu().numpy(), b.arrays["gamma_b"].cpu().numpy()
        assert np.max(np.abs(ga - gb)) <= 1e-12 * np.max(np.abs(gb))


@pytest.mark.parametrize("m,n,m_star", [(13, 53, 25), (4, 16, 5), (6, 20, 4)])
def test_mixed_near_far_wake_split_shapes(cuda, m, n, m_star):
    """The mixed path puts a wake longer than its four FP64 rows into the FP32 stream as two
    lattices that both hold the split row; the workspace must size the stream and the
    partial sums for that (13 x 53 with 25 rows once overran them and left NaN forces).
    Wakes of 5 and 4 rows: one far row, and no far rows at all."""
    c = cases.wing_heave(m=m, n=n, m_star=m_star, n_steps=4)
    out = {}
    for prec in ("fp64", "mixed"):
        dc = _device_case(c, prec, c.n_tstep)
        dc.solve_dynamic(1, c.n_tstep)
        out[prec] = (dc.arrays["gamma_b"][1:].cpu().numpy(), dc.force_total[1:].cpu().numpy())
    assert np.all(np.isfinite(out["mixed"][1]))
    g64, gm = out["fp64"][0], out["mixed"][0]
    assert np.max(np.abs(gm - g64)) < TOL * np.max(np.abs(g64))
    cl64, _ = _coeffs(out["fp64"][1], c)
    clm, _ = _coeffs(out["mixed"][1], c)
    assert np.max(np.abs(clm - cl64)) < TOL * np.max(np.abs(cl64))
