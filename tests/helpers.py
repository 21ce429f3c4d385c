"""Shared helpers: build the same case for the CUDA path and the FP64 oracle."""
from __future__ import annotations

import numpy as np

from flapjax_b200 import cases

RNG_SEED = 1234


def rel_err(a, b):
    """Normwise relative error max|a-b| / max|b| (max|b| floored at 1e-300)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def oracle_uvlm(case: cases.WingCase, mirror=None, gust=None, **kw):
    """``gust``: keyword arguments of a OneMinusCosine flow (gust_length, gust_amplitude,
    ...) in place of the Constant one."""
    from oracle import uvlm_ref as R

    mp, mn = (None, None) if mirror is None else mirror
    uv = R.UVLMRef([(case.m, case.n, case.m_star)], np.arange(case.n + 1), mirror_point=mp, mirror_normal=mn,
                   kernel=case.kernel, r_cut=case.r_cut, free_wake=case.free_wake, **kw)
    ff = R.Constant(case.u_inf, case.rho, True) if gust is None else R.OneMinusCosine(case.u_inf, case.rho, True,
                                                                                     **gust)
    uv.set_design_variables(case.dt, ff, case.zeta_b0, case.hg0)
    return uv, ff


def device_uvlm(case: cases.WingCase, precision="fp64", mirror=None, gust=None, **kw):
    import flapjax_b200 as fj

    kernel = fj.cutoff_kernel(case.r_cut) if case.kernel == "cutoff" else fj.biot_savart_epsilon
    mp, mn = (None, None) if mirror is None else mirror
    uv = fj.UVLM([fj.GridDiscretisation(case.m, case.n, case.m_star)], np.arange(case.n + 1), kernel=kernel,
                 free_wake=case.free_wake, precision=precision, mirror_point=mp, mirror_normal=mn, **kw)
    ff = fj.Constant(case.u_inf, case.rho, True) if gust is None else fj.OneMinusCosine(case.u_inf, case.rho, True,
                                                                                       **gust)
    uv.set_design_variables(dt=case.dt, flowfield=ff, zeta_b0=case.zeta_b0, hg0=case.hg0)
    return uv, ff


def coefficients(force_total, case: cases.WingCase):
    """CL, CD from per-slot total forces (lift/drag axes of the freestream AoA)."""
    a = np.deg2rad(case.alpha_deg)
    e_l = np.array((-np.sin(a), 0.0, np.cos(a)))
    e_d = np.array((np.cos(a), 0.0, np.sin(a)))
    q = 0.5 * case.rho * case.u_mag**2 * case.s_ref
    ft = np.asarray(force_total)
    return ft @ e_l / q, ft @ e_d / q


def oracle_force_total(case_ref):
    return sum(fs.sum(axis=(1, 2)) + fu.sum(axis=(1, 2)) for fs, fu in zip(case_ref.f_steady, case_ref.f_unsteady))
