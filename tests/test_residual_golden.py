"""The time-step residual against the reference's own UVLM.timestep_residual
(aero/uvlm.py:1942-2047), run on the same inputs by tests/golden/make_golden.py (the
reference's source under the NumPy stand-in for jax, with the beam's varphi -> frames map
replaced by the frames themselves): the oracle restatement and the product's residual
(oracle-backed on CPU, device-backed on the GPU) within 1e-11 / 1e-10."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from flapjax_b200.residual import AeroResidual
from oracle import uvlm_ref as R
from oracle import uvlm_residual as RR
from tests.adjoint_oracle import OracleDev

GOLD = Path(__file__).resolve().parent / "golden" / "residual"
CASES = sorted(p.stem for p in GOLD.glob("*.npz"))
_ST = ("gamma_b", "gamma_w", "gamma_b_dot", "zeta_w")


def _load(name):
    with np.load(GOLD / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def _flow(fx, mod):
    if "gust_length" in fx:
        return mod.OneMinusCosine(fx["u_inf"], float(fx["rho"]), True, gust_length=float(fx["gust_length"]),
                                  gust_amplitude=float(fx["gust_amplitude"]), gust_x0=fx["gust_x0"])
    return mod.Constant(fx["u_inf"], float(fx["rho"]), True)


def _inputs(fx):
    qn = {k: [fx[f"q_n_{k}"]] for k in _ST}
    qm = {k: [fx[f"q_nm1_{k}"]] for k in _ST}
    return float(fx["t_n"]), fx["hg_n"], fx["hg_dot_n"], fx["hg_nm1"], qn, qm, fx["f_beam_n"]


def _oracle(fx):
    m, n, ms = (int(v) for v in fx["dims"])
    uv = R.UVLMRef([(m, n, ms)], np.arange(n + 1), kernel=str(fx["kernel"]), r_cut=float(fx["r_cut"]),
                   free_wake=bool(fx["free_wake"]))
    uv.set_design_variables(float(fx["dt"]), _flow(fx, R), fx["zeta_b0"], fx["hg0"])
    return uv


def test_residual_golden_cases_present():
    assert len(CASES) >= 3


@pytest.mark.parametrize("name", CASES)
def test_oracle_residual_matches_reference(name):
    fx = _load(name)
    uv = _oracle(fx)
    want = fx["residual"]
    got = RR.timestep_residual(uv, *_inputs(fx))
    assert np.max(np.abs(got - want)) <= 1e-11 * np.max(np.abs(want))
    ar = AeroResidual(uv, dev=OracleDev(uv.kernel, uv.r_cut, uv.mirror))
    r, _ = ar.vjp(*_inputs(fx), np.zeros_like(want))
    assert np.max(np.abs(r - want)) <= 1e-11 * np.max(np.abs(want))


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_residual_matches_reference(cuda, name):
    import flapjax_b200 as fj

    fx = _load(name)
    m, n, ms = (int(v) for v in fx["dims"])
    kernel = fj.cutoff_kernel(float(fx["r_cut"])) if str(fx["kernel"]) == "cutoff" else fj.biot_savart_epsilon
    uv = fj.UVLM([fj.GridDiscretisation(m, n, ms)], np.arange(n + 1), kernel=kernel, free_wake=bool(fx["free_wake"]),
                 precision="fp64")
    uv.set_design_variables(dt=float(fx["dt"]), flowfield=_flow(fx, fj), zeta_b0=fx["zeta_b0"], hg0=fx["hg0"])
    want = fx["residual"]
    r, _ = AeroResidual(uv, cuda).vjp(*_inputs(fx), np.zeros_like(want))
    assert np.max(np.abs(r - want)) <= 1e-10 * np.max(np.abs(want))
