"""Batched steps and the serving loop: each case's result is the same alone and in the mix.

Tolerances (normwise relative, per field): FP64 1e-12 (only summation grouping differs);
mixed 1e-6 (the FP32 sums are split differently when cases share a launch).
"""
from __future__ import annotations

import numpy as np
import pytest

from flapjax_b200 import cases
from tests.helpers import device_uvlm, rel_err

pytestmark = pytest.mark.gpu

FIELDS = ("gamma_b", "gamma_w", "zeta_w", "f_steady", "f_unsteady", "gamma_b_dot", "alpha")


def _mix():
    return [cases.wing_heave(m=4, n=10, m_star=12, n_steps=6, alpha_deg=3.0, seed=1),
            cases.wing_heave(m=7, n=24, m_star=30, n_steps=6, alpha_deg=6.0, seed=2),
            cases.wing_heave(m=5, n=17, m_star=5, n_steps=6, alpha_deg=1.0, seed=3)]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_batched_steps_match_single_case_runs(cuda, precision, tol):
    from flapjax_b200.serving import BatchStepper

    mix = _mix()
    alone = []
    for c in mix:
        uv, _ = device_uvlm(c, precision)
        alone.append(uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t))
    uvs, dcs = [], []
    for c in mix:
        uv, _ = device_uvlm(c, precision)
        dc = uv.make_device_case(c.n_tstep)
        uv.load_initial(dc, uv.solve_static())
        dc.set_hg(c.hg_t, c.hg_dot_t)
        uvs.append(uv)
        dcs.append(dc)
    st = BatchStepper(8, cuda)
    for i in range(1, mix[0].n_tstep):
        st.step(dcs, [i] * len(dcs), [i > 1] * len(dcs))
    for uv, dc, want in zip(uvs, dcs, alone):
        got = uv._to_case(dc)
        for f in FIELDS:
            for a, b in zip(getattr(got, f), getattr(want, f)):
                assert rel_err(a, b) < tol, (f, rel_err(a, b))


def test_batched_free_wake_and_mirror(cuda):
    """Free-wake and mirrored cases in one batch (FP64, exact up to summation order)."""
    from flapjax_b200.serving import BatchStepper

    mir = (np.zeros(3), np.array([0.0, 1.0, 0.0]))
    mix = [cases.wing_free(m=3, n=8, m_star=6, n_steps=4, seed=4), cases.wing_free(m=4, n=6, m_star=9, n_steps=4, seed=5)]
    outs = []
    for mode in ("alone", "batch"):
        uvs, dcs, res = [], [], []
        for c in mix:
            uv, _ = device_uvlm(c, "fp64", mirror=mir)
            if mode == "alone":
                res.append(uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t))
            else:
                dc = uv.make_device_case(c.n_tstep)
                uv.load_initial(dc, uv.solve_static())
                dc.set_hg(c.hg_t, c.hg_dot_t)
                uvs.append(uv)
                dcs.append(dc)
        if mode == "batch":
            st = BatchStepper(4, cuda)
            for i in range(1, mix[0].n_tstep):
                st.step(dcs, [i, i], [i > 1, i > 1])
            res = [uv._to_case(dc) for uv, dc in zip(uvs, dcs)]
        outs.append(res)
    for got, want in zip(outs[1], outs[0]):
        for f in FIELDS:
            for a, b in zip(getattr(got, f), getattr(want, f)):
                assert rel_err(a, b) < 1e-12, f


@pytest.mark.parametrize("overlap", [True, False])
def test_serving_loop_results_match_alone(cuda, overlap):
    from flapjax_b200.serving import Request, ServingLoop

    rng = np.random.default_rng(0)
    reqs, alone = [], {}
    for k in range(6):
        c = cases.wing_heave(m=int(rng.integers(3, 8)), n=int(rng.integers(6, 20)), m_star=int(rng.integers(4, 20)),
                             n_steps=int(rng.integers(3, 7)), alpha_deg=float(rng.uniform(0, 8)), seed=k)
        uv, _ = device_uvlm(c, "mixed")
        alone[k] = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
        uv2, _ = device_uvlm(c, "mixed")
        reqs.append(Request(uv2, c.hg_t, c.hg_dot_t, arrival=0.01 * k, tag=k))
    loop = ServingLoop(memory_budget=1 << 30, max_active=4, device=cuda, overlap_admission=overlap)
    out = loop.run(reqs, realtime=False)
    summ = out.summary()
    assert summ["case_steps"] == sum(r.hg_t.shape[0] - 1 for r in reqs)
    assert summ["p99_step_ms"] >= summ["p50_step_ms"] > 0
    # serial admission fills the batch 4 at a time; overlapped admission lets cases join
    # as the admission thread finishes them, so the batch may stay narrower
    assert summ["max_active"] == 4 if not overlap else 1 <= summ["max_active"] <= 4
    for k, want in alone.items():
        got = out.results[k]
        for f in FIELDS:
            for a, b in zip(getattr(got, f), getattr(want, f)):
                assert rel_err(a, b) < 1e-6, (k, f, rel_err(a, b))


def test_batched_variable_and_uniform_wakes(cuda):
    """A delta_w case and a uniform-wake case in one batch (FP64): as alone."""
    from flapjax_b200.serving import BatchStepper

    mix = [cases.wing_heave(m=3, n=8, m_star=9, n_steps=5, seed=7), cases.wing_heave(m=4, n=6, m_star=7, n_steps=5)]
    dws = [mix[0].dt * 1.1 ** np.arange(mix[0].m_star), None]
    outs = []
    for mode in ("alone", "batch"):
        uvs, dcs, res = [], [], []
        for c, dw in zip(mix, dws):
            uv, ff = device_uvlm(c, "fp64")
            uv.set_design_variables(dt=c.dt, flowfield=ff, zeta_b0=c.zeta_b0, hg0=c.hg0, delta_w=dw)
            if mode == "alone":
                res.append(uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t))
            else:
                dc = uv.make_device_case(c.n_tstep)
                uv.load_initial(dc, uv.solve_static())
                dc.set_hg(c.hg_t, c.hg_dot_t)
                uvs.append(uv)
                dcs.append(dc)
        if mode == "batch":
            st = BatchStepper(4, cuda)
            for i in range(1, mix[0].n_tstep):
                st.step(dcs, [i, i], [i > 1, i > 1])
            res = [uv._to_case(dc) for uv, dc in zip(uvs, dcs)]
        outs.append(res)
    for got, want in zip(outs[1], outs[0]):
        for f in FIELDS:
            for a, b in zip(getattr(got, f), getattr(want, f)):
                assert rel_err(a, b) < 1e-12, f


@pytest.mark.parametrize("precision,tol", [("fp64", 0.0), ("mixed", 1e-9)])
def test_fsi_iterations_reuse_the_wake_convection(cuda, precision, tol):
    """A fluid-structure loop re-solves one slot with new frames (UVLM.case_solve, as the
    reference beam calls it).  The second and later iterations take the free-wake
    convection (and, mixed, the factors) from the first: the final iterate equals a fresh
    solve of that slot (FP64 bit for bit), with fewer kernel launches per iteration."""
    from flapjax_b200 import _lib

    c = cases.wing_free(m=4, n=10, m_star=12, n_steps=6, seed=2)
    uv, _ = device_uvlm(c, precision)
    case = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    i = 4
    rng = np.random.default_rng(0)
    launches = []
    for it in range(3):
        hg_n = c.hg_t[i].copy()
        hg_n[:, 2, 3] += 1e-3 * rng.normal(size=hg_n.shape[0])  # a structural iterate
        l0 = _lib.load().fj_launch_count()
        uv.case_solve(case, i, hg_n, c.hg_t[i - 1], c.hg_dot_t[i], static=False, horseshoe=False)
        launches.append(_lib.load().fj_launch_count() - l0)
    assert launches[1] < launches[0] and launches[2] == launches[1]
    fresh, _ = device_uvlm(c, precision)
    case2 = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    fresh.case_solve(case2, i, hg_n, c.hg_t[i - 1], c.hg_dot_t[i], static=False, horseshoe=False)
    for f in ("gamma_b", "gamma_w", "zeta_w", "f_steady", "f_unsteady"):
        a, b = getattr(case, f)[0][i], getattr(case2, f)[0][i]
        assert rel_err(a, b) <= tol, (f, rel_err(a, b))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_graph_replay_equals_direct_launches(cuda, precision):
    """fj_step_batched replays a captured graph while the batch's launch signature holds
    and re-captures when it changes (a case leaves the batch, here after step 3); the
    results are bit-identical to direct launches of every kernel."""
    import torch

    from flapjax_b200.serving import BatchStepper, graph_stats

    mix = _mix()
    outs = {}
    for graph in (False, True):
        uvs, dcs = [], []
        for c in mix:
            uv, _ = device_uvlm(c, precision)
            dc = uv.make_device_case(c.n_tstep)
            uv.load_initial(dc, uv.solve_static())
            dc.set_hg(c.hg_t, c.hg_dot_t)
            dc.solve_dynamic(1, 2)  # the factorising first step, outside the batch
            uvs.append(uv)
            dcs.append(dc)
        st = BatchStepper(8, cuda)
        before = graph_stats()
        for i in range(2, mix[0].n_tstep):
            k = len(dcs) if i <= 3 else len(dcs) - 1
            st.step(dcs[:k], [i] * k, [True] * k, graph=graph)
        torch.cuda.synchronize()
        after = graph_stats()
        if graph:
            assert after["captures"] - before["captures"] == 2, (before, after)
            assert after["replays"] - before["replays"] == mix[0].n_tstep - 2 - 2
        else:
            assert after == before
        st.close()
        outs[graph] = [uv._to_case(dc) for uv, dc in zip(uvs, dcs)]
    for a, b in zip(outs[False], outs[True]):
        for f in FIELDS:
            for x, y in zip(getattr(a, f), getattr(b, f)):
                assert np.array_equal(x, y), f
