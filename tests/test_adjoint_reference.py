"""Adjoint gradients against the reference's own forward: tests/golden/gradient/ holds
central differences (h = 1e-6, float64) of the time-mean CL computed by the reference's
UVLM.solve_prescribed_dynamic (its source under the NumPy stand-in for jax) along seeded
directions of zeta_b0.  The hand-written reverse sweep (oracle-backed on CPU,
device-backed on the GPU) must give the same directional derivatives within 1e-6 and the
same objective within 1e-12."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from flapjax_b200 import cases
from tests.adjoint_oracle import OracleAdjoint, coefficient_weights
from tests.helpers import device_uvlm, oracle_uvlm

GOLD = Path(__file__).resolve().parent / "golden" / "gradient"
CASES = sorted(p.stem for p in GOLD.glob("*.npz"))

# the cases the golden generator ran, by name
_BUILD = {
    "gradient_pitch": lambda: cases.wing_pitch(m=3, n=4, m_star=4, n_steps=4, n_ctrl=3, seed=3),
    "gradient_free_cutoff": lambda: cases.wing_free(m=3, n=4, m_star=4, n_steps=3, seed=1),
    "gradient_free_gust": lambda: cases.wing_free(m=3, n=4, m_star=4, n_steps=3, seed=1),
    "gradient_pitch_delta_w": lambda: cases.wing_pitch(m=3, n=4, m_star=5, n_steps=4, n_ctrl=3, seed=3),
    "gradient_free_mirror": lambda: cases.wing_free(m=3, n=4, m_star=4, n_steps=3, seed=1),
}


def _load(name):
    with np.load(GOLD / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def _setup(name):
    fx = _load(name)
    c = _BUILD[name]()
    c.kernel = str(fx["kernel"])
    c.r_cut = float(fx["r_cut"])
    c.free_wake = bool(fx["free_wake"])
    gust = None
    if "gust_length" in fx:
        gust = dict(gust_length=float(fx["gust_length"]), gust_amplitude=float(fx["gust_amplitude"]),
                    gust_x0=fx["gust_x0"])
    dw = fx.get("delta_w")
    mirror = (fx["mirror_point"], fx["mirror_normal"]) if "mirror_point" in fx else None
    return fx, c, gust, dw, mirror


def test_gradient_golden_cases_present():
    assert len(CASES) >= 5


@pytest.mark.parametrize("name", CASES)
def test_oracle_adjoint_matches_reference_differences(name):
    fx, c, gust, dw, mirror = _setup(name)
    uv, ff = oracle_uvlm(c, gust=gust, mirror=mirror)
    if dw is not None:
        uv.set_design_variables(c.dt, ff, c.zeta_b0, c.hg0, delta_w=[dw])
    J, g = OracleAdjoint(uv).gradient(c.hg_t, c.hg_dot_t, coefficient_weights(c, "CL"), checkpoint=2)
    assert abs(J - float(fx["J"])) <= 1e-12 * abs(float(fx["J"]))
    for d, want in zip(fx["directions"], fx["dJ"]):
        assert abs(np.sum(g * d) - want) <= 1e-6 * abs(want)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_adjoint_matches_reference_differences(cuda, name):
    from flapjax_b200.adjoint import PrescribedAdjoint

    fx, c, gust, dw, mirror = _setup(name)
    uv, ff = device_uvlm(c, "fp64", gust=gust, mirror=mirror)
    if dw is not None:
        uv.set_design_variables(dt=c.dt, flowfield=ff, zeta_b0=c.zeta_b0, hg0=c.hg0, delta_w=[dw])
    J, g = PrescribedAdjoint(uv, cuda).gradient(c.hg_t, c.hg_dot_t, coefficient_weights(c, "CL"), checkpoint=2)
    assert abs(J - float(fx["J"])) <= 1e-11 * abs(float(fx["J"]))
    for d, want in zip(fx["directions"], fx["dJ"]):
        assert abs(np.sum(g * d) - want) <= 1e-6 * abs(want)
