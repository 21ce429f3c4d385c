"""A fluid-structure loop with the shape of the reference's fsi_convergence_loop
(structure/beam.py:2656-2674: case_solve, then project_forcing_to_beam, then the
structural update) run against flapjax_b200.UVLM on the device and against the reference's
own UVLM (tests/golden/fsi/*.npz, made with the reference's case_solve and AeroCase under
the NumPy stand-in for jax).  The beam is a typical-section stand-in (tests/fsi_standin.py);
three iterates per step, so iterates 2 and 3 re-solve a slot with new frames from the same
slot n-1 (the free-wake case then reuses the convection of iterate 1).

Tolerances: FP64 within 1e-9 of the reference's projected loads per call (normwise over
the node loads) and of its structural history; mixed within 1e-6."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from tests.fsi_standin import TypicalSection, run_fsi

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "fsi"


def _uvlm(d, precision):
    import flapjax_b200 as fj

    m, n, ms = (int(v) for v in d["dims"])
    kernel = fj.cutoff_kernel(float(d["r_cut"])) if str(d["kernel"]) == "cutoff" else fj.biot_savart_epsilon
    uv = fj.UVLM([fj.GridDiscretisation(m, n, ms)], np.arange(n + 1), kernel=kernel, free_wake=bool(d["free_wake"]),
                 precision=precision, device="cuda:0")
    uv.set_design_variables(dt=float(d["dt"]), flowfield=fj.Constant(d["u_inf"], float(d["rho"]), True),
                            zeta_b0=d["zeta_b0"], hg0=d["hg0"])
    return uv


@pytest.mark.parametrize("name", ["fsi_heave", "fsi_free_cutoff"])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_fsi_loop_matches_reference(cuda, name, precision, tol):
    from flapjax_b200.data_structures import AeroCase

    d = np.load(GOLD / f"{name}.npz")
    uv = _uvlm(d, precision)
    case = AeroCase.initialise(uv.solve_static(), int(d["n_tstep"]))
    rec = []
    case, (x, v, a) = run_fsi(uv, TypicalSection(d["hg0"][:, 1, 3]), case, int(d["n_tstep"]), float(d["dt"]),
                              n_iter=int(d["n_iter"]), record=rec)
    assert len(rec) == d["rec_f"].shape[0]
    for k, (i, it, hg, hgd, f) in enumerate(rec):
        assert (i, it) == (int(d["rec_i"][k]), int(d["rec_it"][k]))
        want = d["rec_f"][k]
        err = np.max(np.abs(f - want)) / np.max(np.abs(want))
        assert err < tol, (i, it, err)
    assert np.max(np.abs(x - d["x"])) < tol * np.max(np.abs(d["x"]))
    err_g = np.max(np.abs(case.gamma_b[0] - d["dyn_gamma_b"])) / np.max(np.abs(d["dyn_gamma_b"]))
    assert err_g < tol
    # the states the coupled adjoint reads (AeroStates ravel order)
    slot = int(d["states_slot"])
    st = case.get_states(slot).ravel()
    assert np.max(np.abs(st - d["states_ravel"])) < tol * np.max(np.abs(d["states_ravel"]))


def test_case_induced_velocity_matches_oracle(cuda):
    """AeroCase.get_v_ind / get_v_tot (aero/data_structures.py:511-531) on the device."""
    from oracle import uvlm_ref as R

    d = np.load(GOLD / "fsi_heave.npz")
    uv = _uvlm(d, "fp64")
    case = uv.solve_static()
    rng = np.random.default_rng(2)
    pts = rng.normal(size=(40, 3)) + [0.5, 3.0, 0.2]
    got = case.get_v_ind(pts)
    want = R.compute_v_ind(pts, [*case.zeta_b, *case.zeta_w], [*case.gamma_b, *case.gamma_w], "epsilon")
    assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))
    tot = case.get_v_tot(pts)
    assert np.allclose(tot - got, d["u_inf"][None], atol=1e-15)


COUPLED = GOLD / "coupled_beam_gust.npz"


@pytest.mark.skipif(not COUPLED.exists(), reason="coupled golden not generated")
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_reference_beam_fsi_sequence(cuda, precision, tol):
    """The reference's geometrically exact beam, coupled to the reference's UVLM, ran its own
    FSI iterations (structure/beam.py:2612-2697) on a clamped, mirrored cantilever with a
    free wake (vortex core 1e-3 c) in a 1-cos gust (tests/golden/make_coupled_golden.py).
    Every case_solve call
    it made is replayed here, in order and with the same frames, through
    flapjax_b200.UVLM.case_solve; the loads project_forcing_to_beam hands back to the beam
    must match the reference's per call (FP64 1e-9, mixed 1e-6 of the call's largest load)."""
    import flapjax_b200 as fj
    from flapjax_b200.data_structures import AeroCase

    d = np.load(COUPLED)
    m, n, ms = (int(v) for v in d["dims"])
    flow = fj.OneMinusCosine(d["u_inf"], float(d["rho"]), True, float(d["gust_length"]), float(d["gust_amplitude"]),
                             gust_x0=d["gust_x0"])
    assert str(d["kernel"]) == "cutoff"
    uv = fj.UVLM([fj.GridDiscretisation(m, n, ms)], np.arange(n + 1), mirror_point=d["mirror_point"],
                 mirror_normal=d["mirror_normal"], kernel=fj.cutoff_kernel(float(d["r_cut"])), free_wake=True,
                 precision=precision, device="cuda:0")
    uv.set_design_variables(dt=float(d["dt"]), flowfield=flow, zeta_b0=d["zeta_b0"], hg0=d["hg0"])
    assert uv.include_unsteady_force == bool(d["include_unsteady_force"])
    init = {k: [d[f"init_{k}"]] for k in ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot",
                                           "gamma_w", "f_steady", "f_unsteady", "alpha")}
    init["n"] = init.pop("nc")
    snap = AeroCase(**init, t=float(d["init_t"]), i_ts=0, **uv._case_meta())
    case = AeroCase.initialise(snap, int(d["n_tstep"]))
    worst = 0.0
    for k in range(d["rec_i"].shape[0]):
        i = int(d["rec_i"][k])
        case = uv.case_solve(case=case, i_ts=i, hg_n=d["rec_hg_n"][k], hg_nm1=d["rec_hg_nm1"][k],
                             hg_dot_n=d["rec_hg_dot_n"][k], static=False, horseshoe=False, cs_ang_n={},
                             cs_ang_nm1={}, cs_vel_n={})
        f = np.asarray(case.project_forcing_to_beam(i, d["rec_hg_n"][k][:, :3, :3], uv.zeta_b0,
                                                    uv.include_unsteady_force))
        want = d["rec_f"][k]
        err = np.max(np.abs(f - want)) / np.max(np.abs(want))
        worst = max(worst, err)
        assert err < tol, (k, i, err)
    last = int(d["rec_i"][-1])
    got = case.gamma_b[0][last]
    assert np.max(np.abs(got - d["dyn_gamma_b"][last])) < tol * np.max(np.abs(d["dyn_gamma_b"][last]))
