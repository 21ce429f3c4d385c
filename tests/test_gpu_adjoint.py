"""Hand-written adjoints on the GPU (FP64).

* fj_vind_vjp against the oracle's VJP of compute_v_ind (1e-10) and central differences;
* fj_lu_solve_t against numpy;
* the device reverse sweep (flapjax_b200.adjoint.PrescribedAdjoint) against the same sweep
  over the oracle (1e-8: the two forwards differ by roundoff) and against central
  differences of the oracle forward in extended precision, h = 1e-6 (1e-6 relative), for
  a lattice direction and for the twist gradient of time-averaged CL and CD.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from flapjax_b200 import cases
from oracle import uvlm_ref as R
from tests.adjoint_oracle import OracleAdjoint, OracleDev, central_difference, coefficient_weights, forward_objective
from tests.helpers import device_uvlm, oracle_uvlm

pytestmark = pytest.mark.gpu


def _lattices(rng):
    z1 = np.zeros((4, 6, 3))
    z1[..., 0] = np.linspace(0, 1, 4)[:, None] + 0.02 * rng.normal(size=(4, 6))
    z1[..., 1] = np.linspace(0, 2, 6)[None, :] + 0.02 * rng.normal(size=(4, 6))
    z1[..., 2] = 0.05 * rng.normal(size=(4, 6))
    z2 = z1 + np.array([1.5, 0.1, 0.2])
    return [(z1, rng.normal(size=(3, 5))), (z2, rng.normal(size=(3, 5)))]


def test_vind_vjp_matches_oracle_and_finite_differences(cuda):
    from flapjax_b200.adjoint import _Dev

    rng = np.random.default_rng(2)
    lats = _lattices(rng)
    tg = rng.normal(size=(40, 3)) * [1.0, 1.5, 0.4] + [0.8, 1.0, 0.0]
    lam = rng.normal(size=(40, 3))
    tb, zb, gb = _Dev(cuda).vjp(tg, lats, lam)
    tb_o, zb_o, gb_o = OracleDev().vjp(tg, lats, lam)
    for got, want in [(tb, tb_o)] + list(zip(zb, zb_o)) + list(zip(gb, gb_o)):
        assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))

    def J(tg_, z1_, g1_, z2_, g2_):
        return float(np.sum(lam * R.compute_v_ind(tg_, [z1_, z2_], [g1_, g2_], R.KERNEL_EPSILON)))

    base = [tg, lats[0][0], lats[0][1], lats[1][0], lats[1][1]]
    grads = [tb, zb[0], gb[0], zb[1], gb[1]]
    h = 1e-6
    for slot, grad in enumerate(grads):
        d = rng.normal(size=base[slot].shape)
        p, m = list(base), list(base)
        p[slot] = base[slot] + h * d
        m[slot] = base[slot] - h * d
        fd = (J(*p) - J(*m)) / (2 * h)
        assert abs(fd - float(np.sum(grad * d))) <= 1e-7 * max(1.0, abs(fd)), slot


def test_vind_vjp_accumulates(cuda):
    """fj_vind_vjp adds into the output cotangents (two calls = twice one call)."""
    import torch

    from flapjax_b200 import _lib

    rng = np.random.default_rng(5)
    (z, g), _ = _lattices(rng)
    tg = rng.normal(size=(17, 3))
    lam = rng.normal(size=(17, 3))
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(cuda)
    tz, tgm, tt, tl = t(z), t(g), t(tg), t(lam)
    outs = [torch.zeros_like(tt), torch.zeros_like(tz), torch.zeros_like(tgm)]
    rows, cols = (C.c_int * 1)(z.shape[0] - 1), (C.c_int * 1)(z.shape[1] - 1)
    n = C.c_size_t()
    _lib.call("fj_vind_vjp_workspace_size", tg.shape[0], rows, cols, 1, 0, C.byref(n))
    ws = torch.empty(n.value, dtype=torch.uint8, device=cuda)
    s = torch.cuda.current_stream(cuda).cuda_stream
    for _ in range(2):
        _lib.call("fj_vind_vjp", tt.data_ptr(), tg.shape[0], (C.c_void_p * 1)(tz.data_ptr()),
                  (C.c_void_p * 1)(tgm.data_ptr()), rows, cols, 1, None, None, _lib.FJ_KERNEL_EPSILON, 0.0,
                  tl.data_ptr(), outs[0].data_ptr(), (C.c_void_p * 1)(outs[1].data_ptr()),
                  (C.c_void_p * 1)(outs[2].data_ptr()), ws.data_ptr(), ws.numel(), s)
    want = OracleDev().vjp(tg, [(z, g)], lam)
    for got, w in zip(outs, (want[0], want[1][0], want[2][0])):
        assert np.max(np.abs(got.cpu().numpy() - 2 * w)) <= 1e-10 * np.max(np.abs(w))


def test_lu_solve_transpose(cuda):
    import torch

    from flapjax_b200 import _lib

    rng = np.random.default_rng(1)
    for n in (5, 70, 300):
        a = rng.normal(size=(n, n)) + 0.05 * n * np.eye(n)
        b = rng.normal(size=n)
        ta = torch.as_tensor(a).to(cuda)
        piv = torch.empty(n, dtype=torch.int32, device=cuda)
        w = C.c_size_t()
        _lib.call("fj_lu_workspace_size", n, C.byref(w))
        ws = torch.empty(w.value, dtype=torch.uint8, device=cuda)
        s = torch.cuda.current_stream(cuda).cuda_stream
        _lib.call("fj_lu_factor", ta.data_ptr(), n, piv.data_ptr(), ws.data_ptr(), ws.numel(), s)
        tb = torch.as_tensor(b).to(cuda)
        _lib.call("fj_lu_solve_t", ta.data_ptr(), n, piv.data_ptr(), tb.data_ptr(), ws.data_ptr(), ws.numel(), s)
        want = np.linalg.solve(a.T, b)
        assert np.max(np.abs(tb.cpu().numpy() - want)) / np.max(np.abs(want)) < 1e-10


@pytest.mark.parametrize("checkpoint", [2, 100])
def test_device_sweep_matches_oracle_sweep(cuda, checkpoint):
    from flapjax_b200.adjoint import PrescribedAdjoint

    c = cases.wing_pitch(m=3, n=4, m_star=4, n_steps=5, n_ctrl=3, seed=3)
    fw = coefficient_weights(c, "CL")
    uv, _ = device_uvlm(c, "fp64")
    J, g = PrescribedAdjoint(uv, cuda).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=checkpoint)
    ref, _ = oracle_uvlm(c)
    J_o, g_o = OracleAdjoint(ref).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=checkpoint)
    assert abs(J - J_o) <= 1e-10 * abs(J_o)
    assert np.max(np.abs(g - g_o)) <= 1e-8 * np.max(np.abs(g_o))
    d = np.random.default_rng(1).normal(size=c.zeta_b0.shape) * 0.1
    fd = central_difference(c, d, fw)
    assert abs(fd - np.sum(g * d)) <= 1e-6 * abs(fd)


@pytest.mark.parametrize("which", ["CL", "CD"])
def test_twist_gradient_matches_finite_differences(cuda, which):
    """Twist gradient of time-averaged CL / CD of a pitching, twisted wing (the adjoint
    configuration at reduced size): device adjoint + twist Jacobian against central
    differences in the twist control angles, h = 1e-6."""
    from flapjax_b200.adjoint import PrescribedAdjoint, twist_jacobian

    c = cases.wing_pitch(m=3, n=6, m_star=5, n_steps=6, n_ctrl=3, seed=4)
    fw = coefficient_weights(c, which)
    uv, _ = device_uvlm(c, "fp64")
    _, g = PrescribedAdjoint(uv, cuda).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=3)
    theta = c.extra["twist_ctrl_rad"]
    ctrl_y = np.linspace(0.0, c.span, len(theta))
    span_y = np.linspace(0.0, c.span, c.n + 1)
    jac = twist_jacobian(c.m, c.n, c.chord, 0.25, ctrl_y, span_y, np.interp(span_y, ctrl_y, theta))
    grad = np.einsum("kmjd,mjd->k", jac, g)
    h = 1e-6
    for k in range(len(theta)):
        # the lattice moves along jac[k] to first order; the second-order part of the
        # twist map enters the central difference at O(h^2)
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        zp = np.asarray(cases.twisted_grid(c.m, c.n, c.chord, 0.25, np.interp(span_y, ctrl_y, tp)), np.longdouble)
        zm = np.asarray(cases.twisted_grid(c.m, c.n, c.chord, 0.25, np.interp(span_y, ctrl_y, tm)), np.longdouble)
        with R.real_type(np.longdouble):
            fd = float((forward_objective(c, zp, fw) - forward_objective(c, zm, fw)) / (2 * h))
        assert abs(fd - grad[k]) <= 1e-6 * max(abs(fd), 1e-2 * np.max(np.abs(grad))), (k, fd, grad[k])


def test_case_factors_copy_matches_direct_factorisation(cuda):
    """The factors an FP64 step solved with equal getrf of the AIC assembled directly
    from that step's lattice."""
    import torch

    from flapjax_b200.adjoint import _Dev

    c = cases.wing_pitch(m=4, n=6, m_star=5, n_steps=3, n_ctrl=3, seed=1)
    uv, _ = device_uvlm(c, "fp64")
    dc = uv.make_device_case(c.n_tstep)
    uv.load_initial(dc, uv.solve_static())
    dc.set_hg(c.hg_t, c.hg_dot_t)
    nb = c.m * c.n
    lu = torch.empty((nb, nb), dtype=torch.float64, device=cuda)
    piv = torch.empty(nb, dtype=torch.int32, device=cuda)
    for i in (1, 2):
        dc.solve_dynamic(i, i + 1)
        dc.copy_factors(lu, piv)
        zb = uv._to_case(dc).zeta_b[0][i]
        rhs = np.random.default_rng(i).normal(size=(c.m, c.n))
        d = _Dev(cuda)
        got = d.solve_t_factors(lu, piv, rhs)
        want = d.solve_t([zb], None, rhs)
        assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


def test_device_sweep_variable_wake(cuda):
    """delta_w on the device forward: the sweep matches the oracle sweep and central
    differences of the extended-precision oracle forward."""
    from flapjax_b200.adjoint import PrescribedAdjoint

    c = cases.wing_pitch(m=3, n=4, m_star=5, n_steps=5, n_ctrl=3, seed=3)
    dw = c.dt * c.u_mag * 1.2 ** np.arange(c.m_star)
    fw = coefficient_weights(c, "CD")
    uv, ff = device_uvlm(c, "fp64")
    uv.set_design_variables(dt=c.dt, flowfield=ff, zeta_b0=c.zeta_b0, hg0=c.hg0, delta_w=dw)
    J, g = PrescribedAdjoint(uv, cuda).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    ref, ffr = oracle_uvlm(c)
    ref.set_design_variables(c.dt, ffr, c.zeta_b0, c.hg0, delta_w=dw)
    J_o, g_o = OracleAdjoint(ref).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    assert abs(J - J_o) <= 1e-10 * abs(J_o)
    assert np.max(np.abs(g - g_o)) <= 1e-8 * np.max(np.abs(g_o))
    d = np.random.default_rng(2).normal(size=c.zeta_b0.shape) * 0.1
    fd = central_difference(c, d, fw, delta_w=dw)
    assert abs(fd - np.sum(g * d)) <= 1e-6 * abs(fd)


def test_cutoff_vind_vjp_matches_oracle(cuda):
    from flapjax_b200 import _lib
    from flapjax_b200.adjoint import _Dev

    rng = np.random.default_rng(7)
    lats = _lattices(rng)
    tg = rng.normal(size=(40, 3)) * [1.0, 1.5, 0.4] + [0.8, 1.0, 0.0]
    lam = rng.normal(size=(40, 3))
    got = _Dev(cuda, _lib.FJ_KERNEL_CUTOFF, 1e-3).vjp(tg, lats, lam)
    want = OracleDev(R.KERNEL_CUTOFF, 1e-3).vjp(tg, lats, lam)
    for a, b in [(got[0], want[0])] + list(zip(got[1], want[1])) + list(zip(got[2], want[2])):
        assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b))


@pytest.mark.parametrize("kernel", ["cutoff", "epsilon"])
def test_device_sweep_free_wake(cuda, kernel):
    """Free wake (the headline workload's kernel: cutoff 1e-3): device sweep against the
    oracle sweep and against extended-precision central differences."""
    from flapjax_b200.adjoint import PrescribedAdjoint

    c = cases.wing_free(m=3, n=5, m_star=5, n_steps=5, seed=2)
    c = cases.WingCase(**{**c.__dict__, "kernel": kernel, "r_cut": 1e-3 if kernel == "cutoff" else 1e-4})
    fw = coefficient_weights(c, "CL")
    uv, _ = device_uvlm(c, "fp64")
    J, g = PrescribedAdjoint(uv, cuda).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    ref, _ = oracle_uvlm(c)
    J_o, g_o = OracleAdjoint(ref).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    assert abs(J - J_o) <= 1e-10 * abs(J_o)
    assert np.max(np.abs(g - g_o)) <= 1e-8 * np.max(np.abs(g_o))
    d = np.random.default_rng(3).normal(size=c.zeta_b0.shape) * 0.1
    fd = central_difference(c, d, fw)
    assert abs(fd - np.sum(g * d)) <= 1e-6 * abs(fd)


def test_device_sweep_mirror(cuda):
    """Mirrored free-wake half-wing: the device sweep (image lattices through fj_vind_vjp
    and the mirrored AIC) against the oracle sweep."""
    from flapjax_b200.adjoint import PrescribedAdjoint

    mir = (np.zeros(3), np.array([0.0, 1.0, 0.0]))
    c = cases.wing_free(m=3, n=5, m_star=5, n_steps=4, seed=2)
    fw = coefficient_weights(c, "CL")
    uv, _ = device_uvlm(c, "fp64", mirror=mir)
    J, g = PrescribedAdjoint(uv, cuda).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    ref, _ = oracle_uvlm(c, mirror=mir)
    J_o, g_o = OracleAdjoint(ref).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    assert abs(J - J_o) <= 1e-10 * abs(J_o)
    assert np.max(np.abs(g - g_o)) <= 1e-8 * np.max(np.abs(g_o))


def test_autograd_wrappers_pass_gradcheck(cuda):
    """The hand-written VJPs behind torch.autograd.Function (fj_vind -> fj_vind_vjp,
    fj_lu_factor/solve -> fj_lu_solve_t) against torch's central differences."""
    import torch

    from flapjax_b200 import _lib
    from flapjax_b200.autograd import dense_solve, induced_velocity

    g = torch.Generator().manual_seed(5)
    R, Cn = 3, 4
    zeta = torch.zeros((R + 1, Cn + 1, 3), dtype=torch.float64)
    zeta[..., 0] = torch.linspace(0.0, 1.0, R + 1)[:, None]
    zeta[..., 1] = torch.linspace(0.0, 2.0, Cn + 1)[None, :]
    zeta += 0.02 * torch.randn(zeta.shape, generator=g, dtype=torch.float64)
    gamma = torch.randn((R, Cn), generator=g, dtype=torch.float64)
    targets = torch.tensor([[0.3, 0.7, 0.4], [1.5, -0.2, 0.3], [0.5, 1.1, -0.6], [-0.4, 2.3, 0.2]],
                           dtype=torch.float64)
    args = [t.to(cuda).requires_grad_(True) for t in (targets, zeta, gamma)]
    for kern, rc in ((_lib.FJ_KERNEL_EPSILON, 0.0), (_lib.FJ_KERNEL_CUTOFF, 1e-3)):
        assert torch.autograd.gradcheck(lambda t, z, gm: induced_velocity(t, z, gm, kern, rc), args, eps=1e-6,
                                        atol=1e-8, rtol=1e-6)
    n = 12
    a = (torch.randn((n, n), generator=g, dtype=torch.float64) + 4 * torch.eye(n, dtype=torch.float64)).to(cuda)
    b = torch.randn(n, generator=g, dtype=torch.float64).to(cuda)
    assert torch.autograd.gradcheck(dense_solve, (a.requires_grad_(True), b.requires_grad_(True)), eps=1e-6,
                                    atol=1e-8, rtol=1e-6)


@pytest.mark.parametrize("builder", ["pitch", "free"])
def test_device_sweep_gust(cuda, builder):
    """A 1-cos gust over the wing: the device sweep (flow evaluated by the CUDA forward, its
    x-derivative in the sweep) against the oracle sweep."""
    from flapjax_b200.adjoint import PrescribedAdjoint

    gust = dict(gust_length=2.0, gust_amplitude=0.1, gust_x0=np.array([-3.0, 0.0, 0.0]))
    c = (cases.wing_pitch(m=3, n=5, m_star=5, n_steps=5, n_ctrl=3, seed=4) if builder == "pitch"
         else cases.wing_free(m=3, n=5, m_star=5, n_steps=4, seed=2))
    fw = coefficient_weights(c, "CL")
    uv, _ = device_uvlm(c, "fp64", gust=gust)
    J, g = PrescribedAdjoint(uv, cuda).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    ref, _ = oracle_uvlm(c, gust=gust)
    J_o, g_o = OracleAdjoint(ref).gradient(c.hg_t, c.hg_dot_t, fw, checkpoint=2)
    assert abs(J - J_o) <= 1e-10 * abs(J_o)
    assert np.max(np.abs(g - g_o)) <= 1e-8 * np.max(np.abs(g_o))


@pytest.mark.parametrize("free_wake", [False, True])
def test_device_sweep_two_surfaces(cuda, free_wake):
    """Wing and tail: the device sweep (both surfaces' lattices in every Biot-Savart VJP,
    the coupled AIC's kept factors in the transpose solve) against the oracle sweep."""
    import flapjax_b200 as fj
    from flapjax_b200.adjoint import PrescribedAdjoint
    from tests.adjoint_oracle import two_surface_case, two_surface_oracle

    surfs, hg0, hg_t, hg_dot_t, wing = two_surface_case(free_wake, n_steps=4)
    fw = coefficient_weights(wing, "CL")
    kernel = fj.cutoff_kernel(wing.r_cut) if wing.kernel == "cutoff" else fj.biot_savart_epsilon
    uv = fj.UVLM([fj.GridDiscretisation(m, n, ms) for m, n, ms, _, _ in surfs], [d for *_, d in surfs],
                 kernel=kernel, free_wake=wing.free_wake, precision="fp64")
    uv.set_design_variables(dt=wing.dt, flowfield=fj.Constant(wing.u_inf, wing.rho, True),
                            zeta_b0=[z for *_, z, _ in surfs], hg0=hg0)
    J, g = PrescribedAdjoint(uv, cuda).gradient(hg_t, hg_dot_t, fw, checkpoint=2)
    J_o, g_o = OracleAdjoint(two_surface_oracle(surfs, hg0, wing)).gradient(hg_t, hg_dot_t, fw, checkpoint=2)
    assert abs(J - J_o) <= 1e-10 * abs(J_o)
    scale = max(np.max(np.abs(a)) for a in g_o)
    for a, b in zip(g, g_o):
        assert np.max(np.abs(a - b)) <= 1e-8 * scale
