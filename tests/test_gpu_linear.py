"""The linearised UVLM on the GPU (aero/linear/linear_uvlm.py): the influence-Jacobian
and many-right-hand-side kernels against the oracle, A, B, C, D against the reference's
own linear model (tests/golden/linear) and against the oracle at larger sizes, and the
linear system against the nonlinear solver for a small heave."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from tests import linear_golden as LG
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


def _lattice(rows, cols, seed):
    rng = np.random.default_rng(seed)
    z = np.zeros((rows + 1, cols + 1, 3))
    z[..., 0] = np.linspace(0.0, 1.0, rows + 1)[:, None]
    z[..., 1] = np.linspace(0.0, 2.0, cols + 1)[None, :]
    z += 0.02 * rng.normal(size=z.shape)
    return z, rng.normal(size=(rows, cols))


@pytest.mark.parametrize("kernel", ["epsilon", "cutoff"])
@pytest.mark.parametrize("mirror", [False, True])
def test_influence_kernels_match_oracle(cuda, kernel, mirror):
    import torch

    from flapjax_b200 import _lib
    from flapjax_b200.linear import _CudaOps
    from tests.linear_cpu_ops import OracleOps

    kid = {"epsilon": _lib.FJ_KERNEL_EPSILON, "cutoff": _lib.FJ_KERNEL_CUTOFF}[kernel]
    rc = 1e-3
    mir = (np.array([0.0, -0.4, 0.0]), np.array([0.0, 1.0, 0.0])) if mirror else None
    z, g = _lattice(3, 4, 1)
    rng = np.random.default_rng(2)
    x = np.stack([rng.uniform(-0.2, 1.2, 7), rng.uniform(-0.2, 2.2, 7), rng.uniform(0.1, 0.6, 7)], axis=1)
    nrm = rng.normal(size=(7, 3))
    gpu, cpu = _CudaOps(cuda, mir), OracleOps(mir)
    for normals in (None, nrm):
        rows = 7 if normals is not None else 21
        for what, width in (("ring", 12), ("vertex", 60)):
            ld, c0 = width + 5, 2
            out = torch.full((rows, ld), float("nan"), dtype=torch.float64, device=cuda)
            want = torch.zeros((rows, ld), dtype=torch.float64)
            tn = None if normals is None else gpu.tensor(normals)
            if what == "ring":
                gpu.ring(out, c0, gpu.tensor(x), tn, gpu.tensor(z), kid, rc)
                cpu.ring(want, c0, cpu.tensor(x), None if normals is None else cpu.tensor(normals), cpu.tensor(z),
                         kid, rc)
            else:
                gpu.vertex(out, c0, gpu.tensor(x), tn, gpu.tensor(z), gpu.tensor(g), kid, rc)
                cpu.vertex(want, c0, cpu.tensor(x), None if normals is None else cpu.tensor(normals), cpu.tensor(z),
                           cpu.tensor(g), kid, rc)
            o = out.cpu().numpy()
            assert np.isnan(o[:, :c0]).all() and np.isnan(o[:, c0 + width:]).all()  # only its block written
            w = want.numpy()[:, c0:c0 + width]
            tol = 1e-12 if what == "ring" else 1e-7  # the oracle's vertex Jacobian is a central difference
            assert rel_err(o[:, c0:c0 + width], w) < tol, (what, normals is None)


def test_lu_solve_many(cuda):
    import torch

    from flapjax_b200 import _lib

    rng = np.random.default_rng(0)
    n, m, ldb = 300, 257, 261
    a = rng.normal(size=(n, n)) + 0.2 * n * np.eye(n)
    b = rng.normal(size=(n, ldb))
    ta = torch.as_tensor(a).to(cuda)
    piv = torch.empty(n, dtype=torch.int32, device=cuda)
    w = C.c_size_t()
    _lib.call("fj_lu_workspace_size", n, C.byref(w))
    wl = torch.empty(w.value, dtype=torch.uint8, device=cuda)
    s = torch.cuda.current_stream(cuda).cuda_stream
    _lib.call("fj_lu_factor", ta.data_ptr(), n, piv.data_ptr(), wl.data_ptr(), wl.numel(), s)
    tb = torch.as_tensor(b).to(cuda)
    _lib.call("fj_lu_solve_many_workspace_size", n, m, C.byref(w))
    ws = torch.empty(w.value, dtype=torch.uint8, device=cuda)
    _lib.call("fj_lu_solve_many", ta.data_ptr(), n, piv.data_ptr(), tb.data_ptr(), m, ldb, ws.data_ptr(), ws.numel(),
              s)
    got = tb.cpu().numpy()
    assert rel_err(got[:, :m], np.linalg.solve(a, b[:, :m])) < 1e-12
    assert np.array_equal(got[:, m:], b[:, m:])
    with pytest.raises(Exception):
        _lib.call("fj_lu_solve_many", ta.data_ptr(), n, piv.data_ptr(), tb.data_ptr(), m, m - 1, ws.data_ptr(),
                  ws.numel(), s)


@pytest.mark.parametrize("n,shift", [(300, 0), (257, 1)])
def test_lti_march_matches_numpy(cuda, n, shift):
    """fj_lti_march (LinearSystem.run's state march): x_i = A x_{i-1} + bu_{i-shift} against
    the same recurrence in NumPy FP64, an even order (16-byte row loads) and an odd one,
    with the input rows strided; a bad shift is refused."""
    import torch

    from flapjax_b200 import _lib

    rng = np.random.default_rng(1)
    nt, ld = 40, n + 3
    a = rng.normal(size=(n, n)) * (0.9 / np.sqrt(n))
    bu = rng.normal(size=(nt, ld))
    x = np.zeros((nt, n))
    x[0] = rng.normal(size=n)
    want = x.copy()
    for i in range(1, nt):
        want[i] = a @ want[i - 1] + bu[i - shift, :n]
    ta, tb, tx = (torch.as_tensor(v).to(cuda) for v in (a, bu, x))
    s = torch.cuda.current_stream(cuda).cuda_stream
    _lib.call("fj_lti_march", ta.data_ptr(), n, tb.data_ptr(), ld, tx.data_ptr(), nt, shift, s)
    assert rel_err(tx.cpu().numpy(), want) < 1e-13
    with pytest.raises(Exception):
        _lib.call("fj_lti_march", ta.data_ptr(), n, tb.data_ptr(), ld, tx.data_ptr(), nt, 2, s)


def test_linear_system_run_matches_oracle(cuda):
    """LinearSystem.run (utils/linear.py:775-822) on the device against the oracle's
    restatement, before and after remove_u_np1."""
    import torch

    from flapjax_b200.linear import LinearSystem
    from oracle.uvlm_linear import LinearSystemRef

    rng = np.random.default_rng(0)
    a = 0.3 * rng.normal(size=(7, 7))
    b, c, d = rng.normal(size=(7, 4)), rng.normal(size=(5, 7)), rng.normal(size=(5, 4))
    u, x0 = rng.normal(size=(9, 4)), rng.normal(size=7)
    ours = LinearSystem(*(torch.as_tensor(z).to(cuda) for z in (a, b, c, d)), 0.1)
    ref = LinearSystemRef(a, b, c, d, 0.1)
    for removed in (False, True):
        if removed:
            ours.remove_u_np1()
            ref.remove_u_np1()
        x, y = ours.run(u, x0)
        xr, yr = ref.run(u, x0)
        assert np.allclose(x.cpu().numpy(), xr, rtol=1e-13, atol=1e-13)
        assert np.allclose(y.cpu().numpy(), yr, rtol=1e-13, atol=1e-13)
    with pytest.raises(ValueError):
        ours.run(u[:, :3])
    with pytest.raises(ValueError):
        ours.run(u, x0[:3])


def _product_uvlm(g, **kw):
    import flapjax_b200 as fj

    m, n, w = (int(v) for v in g["dims"])
    kernel = fj.cutoff_kernel(float(g["r_cut"])) if str(g["kernel"]) == "cutoff" else fj.biot_savart_epsilon
    mir = LG.mirror_of(g)
    mkw = {} if mir is None else dict(mirror_point=mir[0], mirror_normal=mir[1])
    uv = fj.UVLM([fj.GridDiscretisation(m, n, w)], np.arange(n + 1), kernel=kernel, free_wake=bool(g["free_wake"]),
                 **mkw, **kw)
    uv.set_design_variables(dt=float(g["dt"]), flowfield=LG.flow_product(g), zeta_b0=g["zeta_b0"], hg0=g["hg0"],
                            delta_w=g["delta_w"] if "delta_w" in g else None)
    return uv


@pytest.mark.parametrize("name", LG.CASES + LG.VARIABLE)
def test_linear_model_matches_reference(cuda, name):
    """A, B, C, D of the reference's own LinearUVLM (central differences of its step
    functions, h = 1e-6) and its LinearSystem.run over seeded inputs."""
    from flapjax_b200.linear import LinearUVLM

    g = LG.load(name)
    uv = _product_uvlm(g)
    lin = LinearUVLM(uv, uv.solve_static(), str(g["wake_type"]), device=cuda)
    for k in "abcd":
        got = getattr(lin.sys, k).cpu().numpy()
        assert got.shape == g[k].shape, k
        assert np.abs(got - g[k]).max() <= 1e-8 * max(1.0, np.abs(g[k]).max()), k
    x, y, _, _ = lin.run_vectors(g["u_run"], g["x0_run"])
    assert np.allclose(x, g["x_run"], rtol=0, atol=1e-10) and np.allclose(y, g["y_run"], rtol=0, atol=1e-10)


@pytest.mark.parametrize("wake_type,free,kernel,mirror", [("frozen", False, "epsilon", False),
                                                           ("free", True, "cutoff", True)])
def test_linear_model_matches_oracle_larger(cuda, wake_type, free, kernel, mirror):
    """A 4 x 8 wing with a 6-row wake against central differences of the oracle's step."""
    import flapjax_b200 as fj
    from flapjax_b200 import cases
    from flapjax_b200.linear import LinearUVLM
    from oracle import uvlm_linear as OL
    from oracle import uvlm_ref as R

    c = cases.wing_free(m=4, n=8, m_star=6, n_steps=1, seed=3)
    mir = (np.array([0.0, -0.3, 0.0]), np.array([0.0, 1.0, 0.0])) if mirror else None
    rc = 1e-3
    kw = {} if mir is None else dict(mirror_point=mir[0], mirror_normal=mir[1])
    uv = fj.UVLM([fj.GridDiscretisation(c.m, c.n, c.m_star)], np.arange(c.n + 1), free_wake=free,
                 kernel=fj.cutoff_kernel(rc) if kernel == "cutoff" else fj.biot_savart_epsilon, **kw)
    uv.set_design_variables(dt=c.dt, flowfield=fj.Constant(c.u_inf, c.rho, True), zeta_b0=c.zeta_b0, hg0=c.hg0)
    lin = LinearUVLM(uv, uv.solve_static(), wake_type, device=cuda)
    ro = R.UVLMRef([(c.m, c.n, c.m_star)], np.arange(c.n + 1), kernel=kernel, r_cut=rc, free_wake=free, **kw)
    ro.set_design_variables(c.dt, R.Constant(c.u_inf, c.rho), c.zeta_b0, c.hg0)
    want = OL.LinearUVLMRef(ro, ro.solve_static(), wake_type).linearise()
    for k in "abcd":
        got = getattr(lin.sys, k).cpu().numpy()
        w = getattr(want, k)
        assert np.abs(got - w).max() <= 1e-7 * max(1.0, np.abs(w).max()), k


@pytest.mark.parametrize("wake_type,free,kernel", [("frozen", False, "epsilon"), ("free", True, "cutoff")])
def test_linear_model_two_surfaces(cuda, wake_type, free, kernel):
    """A wing and a tail: cross-surface blocks and offsets against the oracle."""
    import flapjax_b200 as fj
    from flapjax_b200.linear import LinearUVLM

    _, _, lin_ref = LG.two_surface_oracle(wake_type, free, kernel)
    want = lin_ref.linearise()
    dims, z0, dofs, hg0, wing = LG.two_surfaces()
    uv = fj.UVLM([fj.GridDiscretisation(*d) for d in dims], dofs, free_wake=free,
                 kernel=fj.cutoff_kernel(1e-3) if kernel == "cutoff" else fj.biot_savart_epsilon)
    uv.set_design_variables(dt=wing.dt, flowfield=fj.Constant(wing.u_inf, wing.rho, True), zeta_b0=z0, hg0=hg0)
    lin = uv.linearise(uv.solve_static(), wake_type)
    assert isinstance(lin, LinearUVLM)
    for k in "abcd":
        got = getattr(lin.sys, k).cpu().numpy()
        w = getattr(want, k)
        assert np.abs(got - w).max() <= 1e-7 * max(1.0, np.abs(w).max()), k


@pytest.mark.parametrize("wake_type,bound_upwash,wake_upwash,unsteady,m_star",
                         [("frozen", True, True, True, 0), ("prescribed", False, True, False, 2)])
def test_linear_model_options(cuda, wake_type, bound_upwash, wake_upwash, unsteady, m_star):
    """No wake rows, and the upwash inputs / unsteady force switched off, against the oracle."""
    import flapjax_b200 as fj
    from flapjax_b200 import cases
    from flapjax_b200.linear import LinearUVLM
    from oracle import uvlm_linear as OL
    from oracle import uvlm_ref as R

    c = cases.wing_heave(m=3, n=4, m_star=m_star, n_steps=1)
    uv = fj.UVLM([fj.GridDiscretisation(c.m, c.n, c.m_star)], np.arange(c.n + 1), kernel=fj.biot_savart_epsilon)
    uv.set_design_variables(dt=c.dt, flowfield=fj.Constant(c.u_inf, c.rho, True), zeta_b0=c.zeta_b0, hg0=c.hg0)
    lin = LinearUVLM(uv, uv.solve_static(), wake_type, bound_upwash, wake_upwash, unsteady, device=cuda)
    ro = R.UVLMRef([(c.m, c.n, c.m_star)], np.arange(c.n + 1))
    ro.set_design_variables(c.dt, R.Constant(c.u_inf, c.rho), c.zeta_b0, c.hg0)
    want = OL.LinearUVLMRef(ro, ro.solve_static(), wake_type, bound_upwash, wake_upwash, unsteady).linearise()
    for k in "abcd":
        got = getattr(lin.sys, k).cpu().numpy()
        w = getattr(want, k)
        assert got.shape == w.shape, k
        assert np.abs(got - w).max() <= 1e-7 * max(1.0, np.abs(w).max()), k


@pytest.mark.parametrize("name", LG.PROJECTED)
def test_linear_model_projections(cuda, name):
    """linearise(input_projection=, output_projection=) against the reference's projected
    linear model (rigid heave-pitch inputs, lift-moment outputs)."""
    from flapjax_b200.linear import LinearUVLM

    g = LG.load(name)
    uv = _product_uvlm(g)
    lin = LinearUVLM(uv, uv.solve_static(), str(g["wake_type"]), device=cuda, skip_linearisation=True)
    ip, op = LG.projections(g)
    sys_ = lin.linearise(input_projection=ip, output_projection=op)
    for k in "abcd":
        got = getattr(sys_, k).cpu().numpy()
        assert got.shape == g[k].shape, k
        assert np.abs(got - g[k]).max() <= 1e-8 * max(1.0, np.abs(g[k]).max()), k


def test_run_with_unflattened_inputs(cuda):
    """LinearUVLM.run as the reference calls it (aero/linear/linear_uvlm.py:869-972):
    per-surface time-batched inputs, a gust flow field turned into upwash perturbations,
    per-surface results and totals; equal to the packed march."""
    import flapjax_b200 as fj
    from flapjax_b200.linear import AeroInputUnflattened, LinearUVLM

    g = LG.load("linear_frozen")
    uv = _product_uvlm(g)
    lin = LinearUVLM(uv, uv.solve_static(), "frozen", device=cuda)
    lay, n_t = lin.layout, 5
    rng = np.random.default_rng(3)
    zb = [1e-3 * rng.normal(size=(n_t,) + np.shape(a)) for a in lin._ref["zeta_b"]]
    zbd = [1e-3 * rng.normal(size=(n_t,) + np.shape(a)) for a in lin._ref["zeta_b"]]
    gust = fj.OneMinusCosine(g["u_inf"], float(g["rho"]), True, gust_length=1.0, gust_amplitude=0.1,
                             gust_x0=np.array([-1.0, 0.0, 0.0]))
    res = lin.run(AeroInputUnflattened(zeta_b=zb, zeta_b_dot=zbd), flowfield=gust)
    t = np.arange(n_t) * lin.dt
    nu_b = [np.stack([gust(z, ti) - gust(z, 0.0) for ti in t]) for z in lin._ref["zeta_b"]]
    nu_w = [np.stack([gust(z, ti) - gust(z, 0.0) for ti in t]) for z in lin._ref["zeta_w"]]
    u = np.concatenate([np.concatenate([a.reshape(n_t, -1) for a in blk], axis=1) for blk in (zb, zbd, nu_b, nu_w)],
                       axis=1)
    x, y, xt, yt = lin.run_vectors(u)
    assert res.n_tstep == n_t and np.allclose(res.t, t)
    assert np.abs(np.concatenate([a.reshape(n_t, -1) for a in res.u_t.nu_w], axis=1) - u[:, -nu_w[0][0].size:]).max() == 0
    got_x = np.concatenate([a.reshape(n_t, -1) for k, _ in lay.x_blocks for a in getattr(res.x_t, k)], axis=1)
    got_y = np.concatenate([a.reshape(n_t, -1) for k, _ in lay.y_blocks for a in getattr(res.y_t, k)], axis=1)
    assert np.array_equal(got_x, x) and np.array_equal(got_y, y)
    tot_y = np.concatenate([a.reshape(n_t, -1) for k, _ in lay.y_blocks for a in getattr(res.y_t_tot, k)], axis=1)
    assert np.allclose(tot_y, yt, rtol=0, atol=1e-14)
    assert np.allclose(res.u_t_tot.zeta_b[0], lin._ref["zeta_b"][0][None] + zb[0], rtol=0, atol=1e-15)
    assert np.abs(res.y_t.f_steady[0]).max() > 0


def test_linear_model_follows_nonlinear_heave(cuda):
    """A heave of 1e-4 chords: the force perturbations of the linear system equal those of
    the nonlinear prescribed-motion solve to second order in the amplitude (cutoff kernel,
    as the linear model's forces; no Gamma_dot filter, as the linear model has none)."""
    import flapjax_b200 as fj
    from flapjax_b200 import cases
    from flapjax_b200.linear import LinearUVLM

    c = cases.wing_heave(m=4, n=8, m_star=12, n_steps=24, amp=1e-4, k=0.4)
    uv = fj.UVLM([fj.GridDiscretisation(c.m, c.n, c.m_star)], np.arange(c.n + 1), kernel=fj.cutoff_kernel(1e-4),
                 gamma_dot_relaxation=1.0)
    uv.set_design_variables(dt=c.dt, flowfield=fj.Constant(c.u_inf, c.rho, True), zeta_b0=c.zeta_b0, hg0=c.hg0)
    st = uv.solve_static()
    dy = uv.solve_prescribed_dynamic(st, c.hg_t, c.hg_dot_t)
    lin = LinearUVLM(uv, st, "prescribed", device=cuda)
    lay = lin.layout
    n_t = c.hg_t.shape[0]
    u = np.zeros((n_t, lin.n_inputs))
    zb = lay.u["zeta_b"]
    zbd = lay.u["zeta_b_dot"]
    z0 = np.asarray(st.zeta_b[0])
    for i in range(n_t):
        zi = np.einsum("jab,ijb->ija", c.hg_t[i][:, :3, :3], c.zeta_b0) + c.hg_t[i][None, :, :3, 3]
        zdi = np.einsum("jab,ijb->ija", c.hg_dot_t[i][:, :3, :3], c.zeta_b0) + c.hg_dot_t[i][None, :, :3, 3]
        u[i, zb[0]:zb[1]] = (zi - z0).ravel()
        u[i, zbd[0]:zbd[1]] = zdi.ravel()
    _, y, _, _ = lin.run_vectors(u)
    nv = (c.m + 1) * (c.n + 1) * 3
    f_lin = (y[:, :nv] + y[:, nv:2 * nv]).reshape(n_t, -1, 3).sum(axis=1)
    f_ref = np.asarray(st.f_steady[0]).sum(axis=(0, 1))
    f_nl = (np.asarray(dy.f_steady[0]) + np.asarray(dy.f_unsteady[0])).sum(axis=(1, 2)) - f_ref
    dz = f_nl[1:, 2]
    assert np.abs(dz).max() > 1e-6  # the heave does load the wing
    assert np.abs(f_lin[1:] - f_nl[1:]).max() < 1e-3 * np.abs(dz).max()
