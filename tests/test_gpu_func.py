"""Function-level entry points against the oracle (FP64, on the GPU).

fj_rhs (aero/uvlm.py:961-983), fj_wake_shed_convect (propagate_surf_wake,
aero/utils.py:400-450), fj_forces (calculate_steady_forcing aero/utils.py:126-223 and the
unsteady term uvlm.py:1086-1103) within 1e-11 normwise; the adjoint twins fj_aic_vjp
(against the oracle-backed transposes and central differences of mu^T A Gamma) and
fj_wake_vjp (against the explicit transpose).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import flapjax_b200 as fj
from flapjax_b200 import _lib, cases
from oracle import uvlm_ref as R
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(dev)


def _ptrs(ts):
    return (C.c_void_p * max(1, len(ts)))(*[t.data_ptr() for t in ts])


def _ints(v):
    return (C.c_int * max(1, len(v)))(*v)


def _stream(dev):
    import torch

    return torch.cuda.current_stream(dev).cuda_stream


def _ws(n, dev):
    import torch

    return torch.empty(max(1, n), dtype=torch.uint8, device=dev)


def _setup(seed=0):
    c = cases.wing_free(m=4, n=7, m_star=5, n_steps=2, seed=seed)
    zb = c.zeta_b0 + np.array([0.0, 0.0, 0.05])
    rng = np.random.default_rng(seed)
    zw = zb[-1][None] + np.arange(c.m_star + 1)[:, None, None] * np.array([0.2, 0.0, 0.02])
    zw = zw + 0.01 * rng.normal(size=zw.shape)
    zw[0] = zb[-1]
    gb = rng.normal(size=(c.m, c.n))
    gw = rng.normal(size=(c.m_star, c.n))
    zbd = 0.1 * rng.normal(size=zb.shape)
    return c, zb, zw, gb, gw, zbd


FLOWS = {
    "constant": (fj.Constant(np.array([1.0, 0.0, 0.08]), 1.225, True),
                 R.Constant(np.array([1.0, 0.0, 0.08]), 1.225, True)),
    "gust": (fj.OneMinusCosine(np.array([1.0, 0.0, 0.08]), 1.225, True, 0.6, 0.1, gust_x0=np.array([-0.5, 0, 0])),
             R.OneMinusCosine(np.array([1.0, 0.0, 0.08]), 1.225, True, 0.6, 0.1, gust_x0=np.array([-0.5, 0, 0]))),
}


@pytest.mark.parametrize("flow", list(FLOWS))
def test_rhs_matches_oracle(cuda, flow):
    ffd, ffo = FLOWS[flow]
    c, zb, zw, gb, gw, zbd = _setup()
    t = 0.37
    cc, nc = R.compute_surf_c(zb), R.compute_surf_nc(zb)
    cdot = R.neighbour_average(zbd, (0, 1))
    want = -np.einsum("ijk,ijk->ij", ffo(cc, t) - cdot + R.compute_v_ind(cc, [zw], [gw], R.KERNEL_EPSILON), nc)
    tz, tg = _t(zw, cuda), _t(gw, cuda)
    n = C.c_size_t()
    np_ = c.m * c.n
    _lib.call("fj_rhs_workspace_size", np_, _ints([c.m_star]), _ints([c.n]), 1, 0, _lib.FJ_PREC_FP64, C.byref(n))
    ws = _ws(n.value, cuda)
    out = _t(np.zeros(np_), cuda)
    fc = ffd.to_c()
    tc, tn, tcd = _t(cc, cuda), _t(nc, cuda), _t(cdot, cuda)  # held: the launches are asynchronous
    _lib.call("fj_rhs", tc.data_ptr(), tn.data_ptr(), tcd.data_ptr(), np_,
              C.byref(fc), t, _ptrs([tz]), _ptrs([tg]), _ints([c.m_star]), _ints([c.n]), 1, None, None,
              _lib.FJ_KERNEL_EPSILON, 0.0, _lib.FJ_PREC_FP64, out.data_ptr(), ws.data_ptr(), ws.numel(), _stream(cuda))
    assert rel_err(out.cpu().numpy().reshape(c.m, c.n), want) < 1e-11
    # static form: no wake, no c_dot
    want0 = -np.einsum("ijk,ijk->ij", ffo(cc, t), nc)
    _lib.call("fj_rhs", tc.data_ptr(), tn.data_ptr(), None, np_, C.byref(fc), t, None, None,
              None, None, 0, None, None, _lib.FJ_KERNEL_EPSILON, 0.0, _lib.FJ_PREC_FP64, out.data_ptr(), ws.data_ptr(),
              ws.numel(), _stream(cuda))
    assert rel_err(out.cpu().numpy().reshape(c.m, c.n), want0) < 1e-14


@pytest.mark.parametrize("free", [False, True])
def test_wake_shed_convect_matches_oracle(cuda, free):
    ffd, ffo = FLOWS["gust"]
    c, zb, zw, gb, gw, zbd = _setup(1)
    t, dt = 0.2, 0.125
    zb_n = zb + np.array([0.01, 0.0, 0.02])

    def v_func(x):
        v = ffo(x, t)
        if free:
            v = v + R.compute_v_ind(x, [zb, zw], [gb, gw], R.KERNEL_EPSILON)
        return v

    zw_want, gw_want = R.propagate_surf_wake(gb, gw, zb_n, zw, None, v_func, dt)
    vconv = R.compute_v_ind(zw[:-1], [zb, zw], [gb, gw], R.KERNEL_EPSILON) if free else None
    zw_out = _t(np.zeros_like(zw), cuda)
    gw_out = _t(np.zeros_like(gw), cuda)
    fc = ffd.to_c()
    held = [_t(zb_n[-1], cuda), _t(gb[-1], cuda), _t(zw, cuda), _t(gw, cuda)]
    tv = None if vconv is None else _t(vconv, cuda)
    _lib.call("fj_wake_shed_convect", *[h.data_ptr() for h in held], None if tv is None else tv.data_ptr(),
              c.n, c.m_star, C.byref(fc), t, dt, zw_out.data_ptr(), gw_out.data_ptr(), _stream(cuda))
    assert rel_err(zw_out.cpu().numpy(), zw_want) < 1e-14
    assert rel_err(gw_out.cpu().numpy(), gw_want) == 0.0


@pytest.mark.parametrize("kernel", [R.KERNEL_EPSILON, R.KERNEL_CUTOFF])
def test_forces_match_oracle(cuda, kernel):
    ffd, ffo = FLOWS["gust"]
    c, zb, zw, gb, gw, zbd = _setup(2)
    t, rc = 0.3, 1e-3
    kid = _lib.FJ_KERNEL_EPSILON if kernel == R.KERNEL_EPSILON else _lib.FJ_KERNEL_CUTOFF

    def v_total(x):
        return ffo(x, t) + R.compute_v_ind(x, [zb, zw], [gb, gw], kernel, None, rc)

    fs_want = R.calculate_steady_forcing([zb], [zbd], [gb], [gw], ffo.rho, v_total)[0]
    gbd = np.random.default_rng(3).normal(size=gb.shape)
    fu_want = R.split_to_vertex(ffo.rho * gbd[..., None] * R.compute_surf_nc(zb), (0, 1))
    rows, cols = _ints([c.m, c.m_star]), _ints([c.n, c.n])
    n = C.c_size_t()
    _lib.call("fj_forces_workspace_size", c.m, c.n, rows, cols, 2, 0, _lib.FJ_PREC_FP64, C.byref(n))
    ws = _ws(n.value, cuda)
    tzb, tzw, tgb, tgw = _t(zb, cuda), _t(zw, cuda), _t(gb, cuda), _t(gw, cuda)
    fs, fu = _t(np.zeros_like(zb), cuda), _t(np.zeros_like(zb), cuda)
    fc = ffd.to_c()
    tzbd, tgw0, tgbd = _t(zbd, cuda), _t(gw[0], cuda), _t(gbd, cuda)
    _lib.call("fj_forces", tzb.data_ptr(), tzbd.data_ptr(), tgb.data_ptr(), tgw0.data_ptr(),
              tgbd.data_ptr(), c.m, c.n, C.byref(fc), t, _ptrs([tzb, tzw]), _ptrs([tgb, tgw]), rows, cols, 2,
              None, None, kid, rc, _lib.FJ_PREC_FP64, fs.data_ptr(), fu.data_ptr(), ws.data_ptr(), ws.numel(),
              _stream(cuda))
    assert rel_err(fs.cpu().numpy(), fs_want) < 1e-11
    assert rel_err(fu.cpu().numpy(), fu_want) < 1e-13


def test_aic_vjp_matches_transposes_and_finite_differences(cuda):
    from flapjax_b200.adjoint import _avg4_T, _normals_T
    from tests.adjoint_oracle import OracleDev

    c, zb, zw, gb, gw, zbd = _setup(4)
    rng = np.random.default_rng(5)
    mu = rng.normal(size=(c.m, c.n))
    n = C.c_size_t()
    _lib.call("fj_aic_vjp_workspace_size", c.m, c.n, C.byref(n))
    ws = _ws(n.value, cuda)
    zbar = _t(np.zeros_like(zb), cuda)
    tzb, tgb, tmu = _t(zb, cuda), _t(gb, cuda), _t(mu, cuda)
    _lib.call("fj_aic_vjp", tzb.data_ptr(), c.m, c.n, tgb.data_ptr(), tmu.data_ptr(),
              _lib.FJ_KERNEL_EPSILON, zbar.data_ptr(), ws.data_ptr(), ws.numel(), _stream(cuda))
    got = zbar.cpu().numpy()
    # the same derivative assembled from the oracle's VJP and the NumPy transposes
    cc, nc = R.compute_surf_c(zb), R.compute_surf_nc(zb)
    V = R.compute_v_ind(cc, [zb], [gb], R.KERNEL_EPSILON)
    cbar, zb_src, _ = OracleDev().vjp(cc, [(zb, gb)], mu[..., None] * nc)
    want = zb_src[0] + _avg4_T(cbar, zb.shape) + _normals_T(zb, mu[..., None] * V)
    assert rel_err(got, want) < 1e-10

    def s(z):
        a = R.compute_aic_solve([R.compute_surf_c(z)], [R.compute_surf_nc(z)], [z], None, R.KERNEL_EPSILON)
        return float(mu.ravel() @ (a @ gb.ravel()))

    # mu^T A Gamma curves on a 1e-3 length scale here (near-core filament terms): the
    # central difference's truncation error is 2e-6 relative at h = 1e-6 and 2e-8 at
    # h = 1e-7 (the same in extended precision, so it is truncation, not roundoff)
    h = 1e-7
    for _ in range(3):
        d = rng.normal(size=zb.shape)
        fd = (s(zb + h * d) - s(zb - h * d)) / (2 * h)
        assert abs(fd - np.sum(got * d)) <= 1e-6 * max(1.0, abs(fd))


def test_wake_vjp_is_the_transpose_of_the_shift(cuda):
    rng = np.random.default_rng(6)
    n, w = 7, 5
    zbar_n = rng.normal(size=(w + 1, n + 1, 3))
    gbar_n = rng.normal(size=(w, n))
    te_z, te_g = rng.normal(size=(n + 1, 3)), rng.normal(size=n)
    zw_prev, gw_prev = rng.normal(size=(w + 1, n + 1, 3)), rng.normal(size=(w, n))
    outs = [_t(a, cuda) for a in (te_z, te_g, zw_prev, gw_prev)]
    tzn, tgn = _t(zbar_n, cuda), _t(gbar_n, cuda)
    _lib.call("fj_wake_vjp", tzn.data_ptr(), tgn.data_ptr(), n, w,
              *[o.data_ptr() for o in outs], _stream(cuda))
    want_te_z = te_z + zbar_n[0]
    want_te_g = te_g + gbar_n[0]
    want_zw = zw_prev.copy()
    want_zw[:-1] += zbar_n[1:]
    want_gw = gw_prev.copy()
    want_gw[:-1] += gbar_n[1:]
    for o, wv in zip(outs, (want_te_z, want_te_g, want_zw, want_gw)):
        assert np.array_equal(o.cpu().numpy(), wv)
