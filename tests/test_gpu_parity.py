"""CUDA path vs the FP64 oracle on the same seeded inputs.

Tolerances: FP64 path within 1e-10 (normwise relative) on circulations; FP32 ("mixed")
Biot-Savart sums within 2e-6 normwise relative per velocity, and force coefficients of
the mixed path within 1e-6 relative of the FP64 path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from flapjax_b200 import _lib, cases
from oracle import uvlm_ref as R
from tests.helpers import coefficients, device_uvlm, oracle_force_total, oracle_uvlm, rel_err

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOL_MIXED_V = 2e-6


def _t(a, dev):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(dev)


# ------------------------------------------------------------------------------------
# kernels
# ------------------------------------------------------------------------------------
def test_kernel_known_answers(cuda):
    """tests/algebra/test_kernels.py:9-98 on the device kernels."""
    import flapjax_b200 as fj

    y = np.array([[0.0, 1.0, 0.0], [0.0, -1.0, 0.0]])
    assert np.all(np.isnan(fj.biot_savart(np.zeros(3), y)))
    assert np.all(np.isnan(fj.biot_savart(np.array([0.0, 1.0, 0.0]), np.array([[0.0, 0.0, 0.0], [0.0, -1.0, 0.0]]))))
    assert not np.all(np.isnan(fj.biot_savart(np.array([0.1, 0.0, 0.0]), y)))
    assert np.allclose(fj.biot_savart_epsilon(np.zeros(3), y), 0.0)
    assert np.allclose(fj.biot_savart_epsilon(np.array([0.0, 1.0, 0.0]), np.array([[0.0, 0.0, 0.0], [0.0, -1.0, 0.0]])), 0.0)
    x = np.array([0.1, 0.0, 0.0])
    assert np.allclose(fj.biot_savart(x, y), fj.biot_savart_epsilon(x, y), rtol=5e-5)
    assert np.allclose(fj.biot_savart_cutoff(np.zeros(3), y), 0.0)
    xo = np.array([1.01e-4, 0.0, 0.0])
    assert np.allclose(fj.biot_savart(xo, y), fj.biot_savart_cutoff(xo, y))
    assert np.allclose(fj.biot_savart_cutoff(np.array([0.99e-4, 0.0, 0.0]), y), 0.0)


def test_kernel_random_pairs_match_oracle(cuda):
    import flapjax_b200 as fj

    rng = np.random.default_rng(7)
    x = rng.normal(size=(4096, 3))
    y = rng.normal(size=(4096, 2, 3))
    for spec, ref in ((fj.biot_savart_epsilon, R.bs_epsilon), (fj.biot_savart, R.bs_plain),
                      (fj.cutoff_kernel(0.05), lambda a, b, c: R.bs_cutoff(a, b, c, 0.05))):
        got = spec(x, y)
        want = ref(x, y[:, 0], y[:, 1])
        assert rel_err(got, want) < 1e-13, spec


# ------------------------------------------------------------------------------------
# compute_v_ind (fj_vind)
# ------------------------------------------------------------------------------------
def _lattices(rng, shapes):
    out = []
    for r, c in shapes:
        z = np.zeros((r + 1, c + 1, 3))
        z[..., 0] = np.linspace(0, 1, r + 1)[:, None] + 0.01 * rng.normal(size=(r + 1, c + 1))
        z[..., 1] = np.linspace(0, 3, c + 1)[None, :] + 0.01 * rng.normal(size=(r + 1, c + 1))
        z[..., 2] = 0.05 * rng.normal(size=(r + 1, c + 1))
        g = rng.normal(size=(r, c))
        out.append((z, g))
    return out


def _fj_vind(dev, targets, lats, kernel, r_cut, precision, mirror=None, ws_fill=None):
    import torch

    from flapjax_b200 import _lib

    tt = _t(targets, dev)
    zs = [_t(z, dev) for z, _ in lats]
    gs = [_t(g, dev) for _, g in lats]
    n = len(lats)
    rows = (C.c_int * n)(*[z.shape[0] - 1 for z, _ in lats])
    cols = (C.c_int * n)(*[z.shape[1] - 1 for z, _ in lats])
    zp = (C.c_void_p * n)(*[z.data_ptr() for z in zs])
    gp = (C.c_void_p * n)(*[g.data_ptr() for g in gs])
    mp = mn = None
    if mirror is not None:
        mp = (C.c_double * 3)(*mirror[0])
        mn = (C.c_double * 3)(*mirror[1])
    nbytes = C.c_size_t()
    _lib.call("fj_vind_workspace_size", targets.shape[0], rows, cols, n, int(mirror is not None), precision,
              C.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    if ws_fill is not None:
        ws.fill_(ws_fill)
    out = torch.empty_like(tt)
    _lib.call("fj_vind", tt.data_ptr(), targets.shape[0], zp, gp, rows, cols, n, mp, mn, kernel, r_cut, precision,
              out.data_ptr(), ws.data_ptr(), ws.numel(), torch.cuda.current_stream(dev).cuda_stream)
    return out.cpu().numpy()


@pytest.mark.parametrize("kernel", ["epsilon", "cutoff"])
@pytest.mark.parametrize("mirror", [False, True])
def test_vind_matches_oracle(cuda, kernel, mirror):
    from flapjax_b200 import _lib

    rng = np.random.default_rng(11)
    lats = _lattices(rng, [(6, 9), (20, 9)])
    # targets: random points, lattice vertices (endpoint coincidence) and filament
    # midpoints (collinear with their own filament)
    z0 = lats[0][0]
    targets = np.concatenate([rng.normal(size=(300, 3)) * [1.0, 2.0, 0.3] + [0.5, 1.5, 0.0], z0.reshape(-1, 3),
                              R.neighbour_average(z0, 0).reshape(-1, 3), R.neighbour_average(z0, 1).reshape(-1, 3)])
    kid = _lib.FJ_KERNEL_EPSILON if kernel == "epsilon" else _lib.FJ_KERNEL_CUTOFF
    r_cut = 1e-3
    mir = (np.array([0.0, -0.2, 0.0]), np.array([0.0, 1.0, 0.0])) if mirror else None
    want = R.compute_v_ind(targets, [z for z, _ in lats], [g for _, g in lats], kernel, mir, r_cut)
    got64 = _fj_vind(cuda, targets, lats, kid, r_cut, _lib.FJ_PREC_FP64, mir)
    # targets on filament lines carry the epsilon regulariser's FP64 rounding noise
    # (|r1 x r2| ~ 1e-16 |r|^2 amplified by 1/(EPSILON |r0|^4)), ~1e-12 of max |v|
    assert rel_err(got64, want) < TOL64
    got32 = _fj_vind(cuda, targets, lats, kid, r_cut, _lib.FJ_PREC_MIXED, mir)
    assert rel_err(got32, want) < TOL_MIXED_V


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_vind_split_below_workspace_bound(cuda, precision):
    """The workspace is sized for the largest split count a shape allows, and the sum
    usually runs with fewer (20 000 targets against a 60 x 200 lattice: about 22 FP64 or
    33 FP32 splits against a bound of 95).  Only the splits that ran may be reduced: the
    workspace starts as NaN bytes (0xFF), so reading an unwritten slab shows."""
    from flapjax_b200 import _lib

    rng = np.random.default_rng(17)
    lats = _lattices(rng, [(60, 200)])
    targets = rng.normal(size=(20000, 3)) * [1.0, 2.0, 0.3] + [0.5, 1.5, 0.0]
    prec = _lib.FJ_PREC_FP64 if precision == "fp64" else _lib.FJ_PREC_MIXED
    got = _fj_vind(cuda, targets, lats, _lib.FJ_KERNEL_EPSILON, 0.0, prec, ws_fill=0xFF)
    assert np.all(np.isfinite(got))
    sub = rng.choice(targets.shape[0], 256, replace=False)
    want = R.compute_v_ind(targets[sub], [lats[0][0]], [lats[0][1]], "epsilon")
    assert rel_err(got[sub], want) < (TOL64 if precision == "fp64" else TOL_MIXED_V)


def test_vind_plain_kernel_fp64(cuda):
    from flapjax_b200 import _lib

    rng = np.random.default_rng(5)
    lats = _lattices(rng, [(5, 7)])
    targets = rng.normal(size=(200, 3)) + [0.5, 1.5, 0.5]
    want = R.compute_v_ind(targets, [lats[0][0]], [lats[0][1]], "plain")
    got = _fj_vind(cuda, targets, lats, _lib.FJ_KERNEL_PLAIN, 0.0, _lib.FJ_PREC_FP64)
    assert rel_err(got, want) < 1e-12


def test_vind_empty_wake_lattice(cuda):
    """A wake with zero rows (m_star = 0) contributes nothing (aero/aic.py:232-233)."""
    from flapjax_b200 import _lib

    rng = np.random.default_rng(3)
    z = np.zeros((1, 6, 3))
    z[0, :, 1] = np.arange(6.0)
    targets = rng.normal(size=(50, 3))
    got = _fj_vind(cuda, targets, [(z, np.zeros((0, 5)))], _lib.FJ_KERNEL_EPSILON, 0.0, _lib.FJ_PREC_FP64)
    assert np.all(got == 0.0)


# ------------------------------------------------------------------------------------
# AIC and the dense solve
# ------------------------------------------------------------------------------------
def _fj_aic(dev, zetas, zetas_w, kernel, r_cut, mirror=None):
    import torch

    from flapjax_b200 import _lib

    n = len(zetas)
    m = (C.c_int * n)(*[z.shape[0] - 1 for z in zetas])
    nn = (C.c_int * n)(*[z.shape[1] - 1 for z in zetas])
    tz = [_t(z, dev) for z in zetas]
    zp = (C.c_void_p * n)(*[z.data_ptr() for z in tz])
    wp = None
    ms = (C.c_int * n)(*([0] * n))
    if zetas_w is not None:
        tw = [_t(z, dev) for z in zetas_w]
        wp = (C.c_void_p * n)(*[z.data_ptr() for z in tw])
        ms = (C.c_int * n)(*[z.shape[0] - 1 for z in zetas_w])
    nb = sum((z.shape[0] - 1) * (z.shape[1] - 1) for z in zetas)
    nbytes = C.c_size_t()
    _lib.call("fj_aic_workspace_size", m, nn, n, C.byref(nbytes))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
    out = torch.empty((nb, nb), dtype=torch.float64, device=dev)
    mp = mn = None
    if mirror is not None:
        mp = (C.c_double * 3)(*mirror[0])
        mn = (C.c_double * 3)(*mirror[1])
    _lib.call("fj_aic_assemble", zp, m, nn, n, wp, ms, mp, mn, kernel, r_cut, out.data_ptr(), ws.data_ptr(),
              ws.numel(), torch.cuda.current_stream(dev).cuda_stream)
    return out.cpu().numpy()


@pytest.mark.parametrize("static", [False, True])
@pytest.mark.parametrize("mirror", [False, True])
def test_aic_matches_oracle(cuda, static, mirror):
    from flapjax_b200 import _lib

    rng = np.random.default_rng(21)
    zs = [z for z, _ in _lattices(rng, [(4, 6), (3, 5)])]
    zs[1] = zs[1] + np.array([2.0, 0.5, 0.3])
    zw = None
    if static:
        zw = []
        for z in zs:
            te = z[-1]
            zw.append(te[None] + np.arange(7)[:, None, None] * np.array([0.2, 0.0, 0.01]))
    mir = (np.array([0.0, -0.5, 0.0]), np.array([0.0, 1.0, 0.0])) if mirror else None
    cs = [R.compute_surf_c(z) for z in zs]
    ns = [R.compute_surf_nc(z) for z in zs]
    want = R.compute_aic_solve(cs, ns, zs, zw, "epsilon", mir)
    got = _fj_aic(cuda, zs, zw, _lib.FJ_KERNEL_EPSILON, 0.0, mir)
    assert rel_err(got, want) < 1e-12


def test_lu_factor_solve_and_mixed(cuda):
    import torch

    from flapjax_b200 import _lib

    rng = np.random.default_rng(4)
    # orders below, at and across the 64-column outer panel, and one whose first panels have
    # more rows than one thread-block cluster holds (2048)
    for n in (1, 7, 64, 65, 333, 1000, 2100):
        a = rng.normal(size=(n, n)) + n * 0.05 * np.eye(n)
        b = rng.normal(size=n)
        want = np.linalg.solve(a, b)
        ta = _t(a, cuda)
        piv = torch.empty(n, dtype=torch.int32, device=cuda)
        nb_ = C.c_size_t()
        _lib.call("fj_lu_workspace_size", n, C.byref(nb_))
        ws = torch.empty(nb_.value, dtype=torch.uint8, device=cuda)
        s = torch.cuda.current_stream(cuda).cuda_stream
        _lib.call("fj_lu_factor", ta.data_ptr(), n, piv.data_ptr(), ws.data_ptr(), ws.numel(), s)
        tb = _t(b, cuda)
        _lib.call("fj_lu_solve", ta.data_ptr(), n, piv.data_ptr(), tb.data_ptr(), ws.data_ptr(), ws.numel(), s)
        assert rel_err(tb.cpu().numpy(), want) < 1e-9 * max(1.0, np.linalg.cond(a) / 1e3)
        # pivots follow LAPACK getrf
        import scipy.linalg

        lu_ref, piv_ref = scipy.linalg.lu_factor(a)
        assert np.array_equal(piv.cpu().numpy(), piv_ref)
        # the factors themselves, to rounding (blocked updates sum in another order)
        _lib.call("fj_lu_factor", ta.copy_(_t(a, cuda)).data_ptr(), n, piv.data_ptr(), ws.data_ptr(), ws.numel(), s)
        assert rel_err(ta.cpu().numpy(), lu_ref) < 1e-11
        # mixed: FP32 factors + FP64 refinement
        nbytes = C.c_size_t()
        _lib.call("fj_solve_mixed_workspace_size", n, C.byref(nbytes))
        wsm = torch.empty(nbytes.value, dtype=torch.uint8, device=cuda)
        ta = _t(a, cuda)
        tx = torch.empty(n, dtype=torch.float64, device=cuda)
        res = torch.empty(1, dtype=torch.float64, device=cuda)
        _lib.call("fj_solve_mixed", ta.data_ptr(), n, _t(b, cuda).data_ptr(), tx.data_ptr(), 1, res.data_ptr(),
                  wsm.data_ptr(), wsm.numel(), s)
        assert rel_err(tx.cpu().numpy(), want) < 1e-11
        assert float(res.cpu()) < 1e-12


# ------------------------------------------------------------------------------------
# full solves through the UVLM API
# ------------------------------------------------------------------------------------
def _compare_case(got, want, tol, fields=("gamma_b", "gamma_w", "zeta_w", "f_steady", "f_unsteady", "gamma_b_dot")):
    for f in fields:
        for a, b in zip(getattr(got, f), getattr(want, f)):
            assert rel_err(a, b) < tol, (f, rel_err(a, b))


@pytest.mark.parametrize("horseshoe", [False, True])
def test_static_solve_matches_oracle(cuda, horseshoe):
    c = cases.wing_heave(m=5, n=12, m_star=15, n_steps=1)
    uv, _ = device_uvlm(c)
    ur, _ = oracle_uvlm(c)
    got = uv.solve_static(horseshoe=horseshoe)
    want = ur.solve_static(horseshoe=horseshoe)
    for f in ("gamma_b", "gamma_w", "zeta_w", "f_steady", "alpha", "c", "nc", "zeta_b"):
        for a, b in zip(getattr(got, f), getattr(want, f)):
            assert rel_err(a, b[0]) < TOL64, f


def test_dynamic_heave_matches_oracle(cuda):
    c = cases.wing_heave(m=4, n=10, m_star=12, n_steps=12)
    uv, _ = device_uvlm(c)
    ur, _ = oracle_uvlm(c)
    got = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    want = ur.solve_prescribed_dynamic(ur.solve_static(), c.hg_t, c.hg_dot_t)
    _compare_case(got, want, TOL64)
    assert rel_err(got.t, want.t) == 0.0
    for a, b in zip(got.alpha, want.alpha):
        assert rel_err(a, b) < TOL64


def test_dynamic_pitch_twist_matches_oracle(cuda):
    c = cases.wing_pitch(m=4, n=8, m_star=10, n_steps=10, n_ctrl=5)
    uv, _ = device_uvlm(c)
    ur, _ = oracle_uvlm(c)
    got = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    want = ur.solve_prescribed_dynamic(ur.solve_static(), c.hg_t, c.hg_dot_t)
    _compare_case(got, want, TOL64)


def test_free_wake_matches_oracle(cuda):
    c = cases.wing_free(m=4, n=12, m_star=16, n_steps=10)
    uv, _ = device_uvlm(c)
    ur, _ = oracle_uvlm(c)
    got = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    want = ur.solve_prescribed_dynamic(ur.solve_static(), c.hg_t, c.hg_dot_t)
    _compare_case(got, want, TOL64)


def test_mirror_matches_oracle(cuda):
    c = cases.wing_heave(m=4, n=8, m_star=10, n_steps=6)
    mir = (np.zeros(3), np.array([0.0, 1.0, 0.0]))
    uv, _ = device_uvlm(c, mirror=mir)
    ur, _ = oracle_uvlm(c, mirror=mir)
    got = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    want = ur.solve_prescribed_dynamic(ur.solve_static(), c.hg_t, c.hg_dot_t)
    _compare_case(got, want, TOL64)


def test_full_heave_config_fp64_and_mixed(cuda):
    """8 x 32 wing, W = 64, 50 heave steps: FP64 path vs oracle (1e-10 on gamma) and
    the mixed path's CL/CD vs the FP64 path (1e-6 relative)."""
    c = cases.wing_heave()
    ur, _ = oracle_uvlm(c)
    want = ur.solve_prescribed_dynamic(ur.solve_static(), c.hg_t, c.hg_dot_t)
    uv, _ = device_uvlm(c, "fp64")
    got = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    _compare_case(got, want, TOL64, fields=("gamma_b", "gamma_w"))
    um, _ = device_uvlm(c, "mixed")
    gm = um.solve_prescribed_dynamic(um.solve_static(), c.hg_t, c.hg_dot_t)
    cl64, cd64 = coefficients(got.force_total, c)
    clm, cdm = coefficients(gm.force_total, c)
    assert np.max(np.abs(clm - cl64) / np.abs(cl64)) < 1e-6
    assert np.max(np.abs(cdm - cd64)) / np.max(np.abs(cd64)) < 1e-6
    clr, _ = coefficients(oracle_force_total(want), c)
    assert np.max(np.abs(cl64 - clr) / np.abs(clr)) < TOL64


@pytest.mark.parametrize("free", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_variable_wake_matches_oracle(cuda, free, precision):
    """delta_w (propagate_surf_wake's re-discretisation, aero/utils.py:452-491): wake
    segments growing 12 % per row; FP64 within 1e-10 of the oracle, mixed within 1e-4."""
    if free:
        c = cases.wing_free(m=4, n=10, m_star=14, n_steps=8)
    else:
        c = cases.wing_heave(m=4, n=10, m_star=14, n_steps=8)
    dw = c.dt * c.u_mag * 1.12 ** np.arange(c.m_star)
    uv, ff = device_uvlm(c, precision)
    uv.set_design_variables(dt=c.dt, flowfield=ff, zeta_b0=c.zeta_b0, hg0=c.hg0, delta_w=dw)
    ur, ffr = oracle_uvlm(c)
    ur.set_design_variables(c.dt, ffr, c.zeta_b0, c.hg0, delta_w=dw)
    got = uv.solve_prescribed_dynamic(uv.solve_static(), c.hg_t, c.hg_dot_t)
    want = ur.solve_prescribed_dynamic(ur.solve_static(), c.hg_t, c.hg_dot_t)
    if precision == "fp64":
        _compare_case(got, want, TOL64)
    else:
        _compare_case(got, want, 1e-4, fields=("gamma_b", "gamma_w", "zeta_w", "f_steady"))
    # the wake really follows delta_w: first-column segment lengths at the last step
    seg = np.linalg.norm(np.diff(got.zeta_w[0][-1][:, 0], axis=0), axis=-1)
    assert np.all(seg[1:] > seg[:-1])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replayed_steps_match_direct_launches(cuda, precision):
    """A run of steps replayed from one captured step graph gives the same slots,
    bit for bit, as launching every step directly (free wake, so every kernel runs)."""
    import torch

    c = cases.wing_free(m=4, n=10, m_star=12, n_steps=9)
    outs = []
    for graph in (False, True):
        uv, _ = device_uvlm(c, precision)
        dc = uv.make_device_case(c.n_tstep)
        uv.load_initial(dc, uv.solve_static())
        dc.set_hg(c.hg_t, c.hg_dot_t)
        launches0 = _lib.load().fj_launch_count()
        dc.solve_dynamic(1, c.n_tstep, graph=graph)
        torch.cuda.synchronize()
        outs.append((dc.host_arrays(), _lib.load().fj_launch_count() - launches0))
    (a, na), (b, nb) = outs
    for f in ("gamma_b", "gamma_w", "zeta_w", "f_steady", "f_unsteady", "gamma_b_dot", "alpha"):
        assert np.array_equal(a[f], b[f]), f
    assert np.array_equal(a["t"], b["t"]) and np.array_equal(a["force_total"], b["force_total"])
    # the launch counter counts the kernels the replays executed (plus the graph's two)
    assert nb >= na


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cached_step_graph_across_calls(cuda, precision):
    """Consecutive calls on one workspace replay the step graph captured by the first
    (the chunked calls of a streaming caller); the slots equal one direct-launch run bit
    for bit, and a second case on another workspace gets its own graph."""
    import torch

    c = cases.wing_free(m=4, n=10, m_star=12, n_steps=13)
    got = []
    for chunks in ([(1, c.n_tstep)], [(1, 2), (2, 5), (5, 9), (9, c.n_tstep)]):
        for graph in ((False,) if len(chunks) == 1 else (True,)):
            uv, _ = device_uvlm(c, precision)
            dc = uv.make_device_case(c.n_tstep)
            uv.load_initial(dc, uv.solve_static())
            dc.set_hg(c.hg_t, c.hg_dot_t)
            other = uv.make_device_case(c.n_tstep)  # interleaved calls on another workspace
            uv.load_initial(other, uv.solve_static())
            other.set_hg(c.hg_t, c.hg_dot_t)
            for i0, i1 in chunks:
                dc.solve_dynamic(i0, i1, reuse_factors=i0 > 1, graph=graph)
                other.solve_dynamic(i0, i1, reuse_factors=i0 > 1, graph=graph)
            torch.cuda.synchronize()
            got.append((dc.host_arrays(), other.host_arrays()))
    (a, _), (b, b2) = got
    for f in ("gamma_b", "gamma_w", "zeta_w", "f_steady", "f_unsteady", "gamma_b_dot", "alpha"):
        assert np.array_equal(a[f], b[f]), f
        assert np.array_equal(b[f], b2[f]), f


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cached_step_graph_not_replayed_for_another_length(cuda, precision):
    """A shorter case on the workspace of a longer one (the same address, as a caching
    allocator hands out after a free) has the same step table address but its slot counter
    elsewhere: it captures its own step graph.  Its slots equal a direct-launch run on a
    workspace of its own, bit for bit.  The longer case stays alive, so its graph's
    pointers stay valid memory whatever is replayed."""
    import torch

    long_c = cases.wing_free(m=4, n=10, m_star=12, n_steps=20)
    short_c = cases.wing_free(m=4, n=10, m_star=12, n_steps=10)
    uv, _ = device_uvlm(long_c, precision)
    dl = uv.make_device_case(long_c.n_tstep)
    uv.load_initial(dl, uv.solve_static())
    dl.set_hg(long_c.hg_t, long_c.hg_dot_t)
    dl.solve_dynamic(1, long_c.n_tstep, graph=True)
    got = []
    for shared in (True, False):
        uv_s, _ = device_uvlm(short_c, precision)
        ds = uv_s.make_device_case(short_c.n_tstep)
        if shared:
            assert ds.ws.numel() <= dl.ws.numel()
            ds.ws = dl.ws[: ds.ws.numel()]
        uv_s.load_initial(ds, uv_s.solve_static())
        ds.set_hg(short_c.hg_t, short_c.hg_dot_t)
        ds.solve_dynamic(1, short_c.n_tstep, graph=shared)
        torch.cuda.synchronize()
        got.append(ds.host_arrays())
    for f in ("gamma_b", "gamma_w", "zeta_w", "f_steady", "f_unsteady", "gamma_b_dot", "alpha"):
        assert np.array_equal(got[0][f], got[1][f]), f
