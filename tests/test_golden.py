"""Golden vectors produced by the reference's own UVLM code (tests/golden/make_golden.py).

CPU: the FP64 oracle reproduces every field of every case (pins the oracle).
GPU: the CUDA path reproduces them, FP64 within 1e-10 and the mixed path within the
FP32 sums' error (1e-5 on circulations, normwise).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import uvlm_ref as R
from tests.helpers import rel_err

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("*.npz"))
FIELDS = ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
          "f_unsteady", "alpha")


def load(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def _surfaces(fx):
    out = []
    for i in range(int(fx["n_surf"])):
        m, n, ms = (int(v) for v in fx[f"surf{i}_dims"])
        out.append((m, n, ms, fx[f"surf{i}_zeta_b0"], fx[f"surf{i}_dof"]))
    return out


def _flow(fx, mod):
    if str(fx["flow_kind"]) == "constant":
        return mod.Constant(fx["u_inf"], float(fx["rho"]), True)
    return mod.OneMinusCosine(fx["u_inf"], float(fx["rho"]), True, gust_length=float(fx["gust_length"]),
                              gust_amplitude=float(fx["gust_amplitude"]))


def _delta_w(fx):
    dws = [fx.get(f"surf{i}_delta_w") for i in range(int(fx["n_surf"]))]
    return None if all(d is None for d in dws) else dws


def _polars(fx, make):
    """Per-surface strip polars from the fixture's tables (None where a surface has none),
    built with ``make(alpha, cl, cd, cm)``; (polars, circulation scale)."""
    n_surf = int(fx["n_surf"])
    if not any(f"surf{i}_polars" in fx for i in range(n_surf)):
        return None, 0.0
    out = []
    for i in range(n_surf):
        t = fx.get(f"surf{i}_polars")
        out.append(None if t is None else [make(r[:, 0], r[:, 1], r[:, 2], r[:, 3]) for r in t])
    return out, float(fx["polar_circulation_scale"])


def _mirror(fx):
    return (fx["mirror_point"], fx["mirror_normal"]) if "mirror_point" in fx else (None, None)


def _compare(get, fx, prefix, tol, fields=FIELDS):
    for f in fields:
        for i in range(int(fx["n_surf"])):
            want = fx[f"{prefix}_{f}_{i}"]
            got = np.asarray(get(f)[i])
            assert got.shape == want.shape, (f, got.shape, want.shape)
            err = rel_err(got, want) if np.max(np.abs(want)) > 0 else float(np.max(np.abs(got)))
            assert err <= tol, (prefix, f, i, err)


def test_golden_cases_present():
    assert len(CASES) >= 10


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_golden(name):
    fx = load(name)
    surfs = _surfaces(fx)
    mp, mn = _mirror(fx)
    pol, pscale = _polars(fx, R.TabulatedPolar)
    uv = R.UVLMRef([(m, n, ms) for m, n, ms, _, _ in surfs], [d for *_, d in surfs], mirror_point=mp,
                   mirror_normal=mn, kernel=str(fx["kernel"]), r_cut=float(fx["r_cut"]),
                   free_wake=bool(fx["free_wake"]), gamma_dot_relaxation=float(fx["gamma_dot_relaxation"]),
                   polars=pol, polar_circulation_scale=pscale)
    uv.set_design_variables(float(fx["dt"]), _flow(fx, R), [z for *_, z, _ in surfs], fx["hg0"],
                            delta_w=_delta_w(fx))
    st = uv.solve_static(horseshoe=bool(fx["horseshoe"]))
    # most fields agree bit for bit; gamma_b_dot = dGamma / dt magnifies the last-digit
    # differences of the free-wake sums (NumPy einsum grouping), hence 1e-11
    _compare(lambda f: [a[0] for a in getattr(st, f)], fx, "static",
             1e-11, fields=[f for f in FIELDS if f"static_{f}_0" in fx])
    if "hg_t" in fx:
        dy = uv.solve_prescribed_dynamic(st, fx["hg_t"], fx["hg_dot_t"])
        _compare(lambda f: getattr(dy, f), fx, "dyn", 1e-11)
        assert np.array_equal(dy.t, fx["dyn_t"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", CASES)
def test_cuda_matches_reference_golden(cuda, name, precision):
    import flapjax_b200 as fj

    fx = load(name)
    surfs = _surfaces(fx)
    mp, mn = _mirror(fx)
    kernel = {"epsilon": fj.biot_savart_epsilon, "plain": fj.biot_savart,
              "cutoff": fj.cutoff_kernel(float(fx["r_cut"]))}[str(fx["kernel"])]
    pol, pscale = _polars(fx, fj.TabulatedPolar)
    uv = fj.UVLM([fj.GridDiscretisation(m, n, ms) for m, n, ms, _, _ in surfs], [d for *_, d in surfs],
                 mirror_point=mp, mirror_normal=mn, kernel=kernel, free_wake=bool(fx["free_wake"]),
                 gamma_dot_relaxation=float(fx["gamma_dot_relaxation"]), precision=precision, polars=pol,
                 polar_circulation_scale=pscale)
    uv.set_design_variables(dt=float(fx["dt"]), flowfield=_flow(fx, fj), zeta_b0=[z for *_, z, _ in surfs],
                            hg0=fx["hg0"], delta_w=_delta_w(fx))
    tol_b = 1e-10 if precision == "fp64" else 1e-5
    st = uv.solve_static(horseshoe=bool(fx["horseshoe"]))
    _compare(lambda f: getattr(st, f), fx, "static", tol_b,
             fields=[f for f in ("gamma_b", "gamma_w", "zeta_w", "f_steady", "alpha", "c", "nc")
                     if f"static_{f}_0" in fx])
    if "hg_t" in fx:
        dy = uv.solve_prescribed_dynamic(st, fx["hg_t"], fx["hg_dot_t"])
        fields = ("gamma_b", "gamma_w", "zeta_w", "f_steady", "alpha")
        _compare(lambda f: getattr(dy, f), fx, "dyn", tol_b if precision == "fp64" else 1e-4, fields=fields)
        # f_unsteady = rho gamma_dot n inherits gamma_dot's 1/dt: measured against the
        # total force scale
        for i in range(int(fx["n_surf"])):
            scale = np.max(np.abs(fx[f"dyn_f_steady_{i}"])) + np.max(np.abs(fx[f"dyn_f_unsteady_{i}"]))
            err = np.max(np.abs(dy.f_unsteady[i] - fx[f"dyn_f_unsteady_{i}"])) / scale
            assert err < (tol_b if precision == "fp64" else 1e-5), ("f_unsteady", i, err)
        # gamma_dot = dGamma/dt: its error is measured against the circulation scale per
        # step, max|Gamma| / dt (the FP32 error of Gamma enters divided by dt)
        for i in range(int(fx["n_surf"])):
            scale = np.max(np.abs(fx[f"dyn_gamma_b_{i}"])) / float(fx["dt"])
            err = np.max(np.abs(dy.gamma_b_dot[i] - fx[f"dyn_gamma_b_dot_{i}"])) / scale
            assert err < (tol_b if precision == "fp64" else 1e-5), ("gamma_b_dot", i, err)
        assert rel_err(dy.t, fx["dyn_t"]) == 0.0
