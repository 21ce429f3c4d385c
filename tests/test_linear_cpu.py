"""The linearised UVLM on the CPU: the oracle against the reference's own linear model
(tests/golden/linear, FD Jacobians of the reference's LinearUVLM step functions), and the
device assembly's chain rule and block bookkeeping with CPU stand-ins for its device
operations (tests/linear_cpu_ops.py)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from tests import linear_golden as LG


def _oracle(g):
    from oracle import uvlm_linear as OL
    from oracle import uvlm_ref as R

    m, n, w = (int(v) for v in g["dims"])
    kern = {"epsilon": R.KERNEL_EPSILON, "cutoff": R.KERNEL_CUTOFF}[str(g["kernel"])]
    mir = LG.mirror_of(g)
    kw = {} if mir is None else dict(mirror_point=mir[0], mirror_normal=mir[1])
    uv = R.UVLMRef([(m, n, w)], np.arange(n + 1), kernel=kern, r_cut=float(g["r_cut"]),
                   free_wake=bool(g["free_wake"]), **kw)
    uv.set_design_variables(float(g["dt"]), LG.flow_oracle(g), g["zeta_b0"], g["hg0"],
                            delta_w=g["delta_w"] if "delta_w" in g else None)
    return OL.LinearUVLMRef(uv, uv.solve_static(), str(g["wake_type"]))


@pytest.mark.parametrize("name", LG.CASES + LG.VARIABLE)
def test_oracle_step_matches_reference(name):
    g = LG.load(name)
    lin = _oracle(g)
    u0, x0 = lin.reference_vectors()
    x1, y0 = lin.step(u0, x0)
    assert np.allclose(x1, g["x_ref"], rtol=0, atol=1e-13)
    assert np.allclose(y0, g["y_ref"], rtol=0, atol=1e-13)
    # the nonlinear step away from the reference point
    up, xp = u0.copy(), x0.copy()
    for blocks, vec, kind in ((lin.u_blocks, up, "u"), (lin.x_blocks, xp, "x")):
        off = 0
        for k, tmpl in blocks:
            size = sum(a.size for a in tmpl)
            key = {"u": {"zeta_b": "zeta_b_np1_vec", "zeta_b_dot": "zeta_b_dot_np1_vec", "nu_b": "nu_b_np1_vec",
                         "nu_w": "nu_w_np1_vec"},
                   "x": {"gamma_b": "gamma_b_n_vec", "gamma_w": "gamma_w_n_vec", "gamma_b_nm1": "gamma_b_nm1_vec",
                         "zeta_w": "zeta_w_n_vec", "zeta_b": "zeta_b_n_vec"}}[kind][k]
            if f"pert_{key}" in g:
                vec[off:off + size] = g[f"pert_{key}"]
            off += size
    x1p, y0p = lin.step(up, xp)
    assert np.allclose(x1p, g["x_pert"], rtol=0, atol=1e-12)
    assert np.allclose(y0p, g["y_pert"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", LG.CASES + LG.VARIABLE)
def test_oracle_jacobians_match_reference(name):
    """Central differences of the oracle's step against those of the reference's step (both
    h = 1e-6): agreement to the differencing noise."""
    g = LG.load(name)
    sys_ = _oracle(g).linearise()
    for k in "abcd":
        assert np.abs(getattr(sys_, k) - g[k]).max() <= 1e-8 * max(1.0, np.abs(g[k]).max()), k
    x, y = sys_.run(g["u_run"], g["x0_run"])
    assert np.allclose(x, g["x_run"], rtol=0, atol=1e-10)
    assert np.allclose(y, g["y_run"], rtol=0, atol=1e-10)


@pytest.mark.parametrize("name", LG.CASES + LG.VARIABLE)
def test_assembly_chain_rule_matches_reference(name):
    """The device assembly's chain rule with the oracle standing in for the device
    operations: A, B, C, D equal the reference's Jacobians, every block (zero blocks
    included: the reference does not differentiate them)."""
    from flapjax_b200 import linear as L
    from tests.linear_cpu_ops import OracleOps

    g = LG.load(name)
    cfg = LG.config(g, LG.flow_product(g))
    lay = L._Layout(LG.dims(g), cfg["wake_type"], True, True, True)
    rs, ro = L._assemble(OracleOps(LG.mirror_of(g)), lay, LG.reference(g), cfg)
    ns = lay.n_states
    got = {"a": rs[:, :ns], "b": rs[:, ns:], "c": ro[:, :ns], "d": ro[:, ns:]}
    for k in "abcd":
        want = g[k]
        assert got[k].shape == want.shape, k
        assert np.abs(got[k].numpy() - want).max() <= 1e-8 * max(1.0, np.abs(want).max()), k


def test_assembly_two_surfaces_against_oracle():
    """Two surfaces (free wake, cutoff kernel): the cross-surface blocks and every offset
    of the assembly against central differences of the oracle's step."""
    from flapjax_b200 import _lib
    from flapjax_b200 import linear as L
    from flapjax_b200.flowfields import Constant
    from tests.linear_cpu_ops import OracleOps

    uv, st, lin = LG.two_surface_oracle("free", True, "cutoff")
    want = lin.linearise()
    dims, *_, wing = LG.two_surfaces()
    ref = {k: [a[0] for a in getattr(st, k)] for k in ("zeta_b", "zeta_w", "gamma_b", "gamma_w")}
    cfg = {"wake_type": "free", "free_wake": True, "kernel": _lib.FJ_KERNEL_CUTOFF, "r_cut": 1e-3,
           "force_r_cut": 1e-3, "dt": wing.dt, "rho": wing.rho, "flowfield": Constant(wing.u_inf, wing.rho, True),
           "t": 0.0, "bound_upwash": True, "wake_upwash": True, "unsteady_force": True}
    lay = L._Layout(dims, "free", True, True, True)
    rs, ro = L._assemble(OracleOps(None), lay, ref, cfg)
    ns = lay.n_states
    got = {"a": rs[:, :ns], "b": rs[:, ns:], "c": ro[:, :ns], "d": ro[:, ns:]}
    for k in "abcd":
        w = getattr(want, k)
        assert np.abs(got[k].numpy() - w).max() <= 1e-8 * max(1.0, np.abs(w).max()), k


@pytest.mark.parametrize("wake_type,bound_upwash,wake_upwash,unsteady,m_star",
                         [("frozen", False, False, False, 3), ("prescribed", True, False, True, 3),
                          ("frozen", True, True, True, 0), ("prescribed", False, True, False, 0),
                          ("free", True, True, True, 1)])
def test_assembly_options_against_oracle(wake_type, bound_upwash, wake_upwash, unsteady, m_star):
    """The upwash inputs and the unsteady force switched off, and wakes of zero and one
    row: the assembly against central differences of the oracle's step (2 x 2 wing)."""
    from flapjax_b200 import _lib, cases
    from flapjax_b200 import linear as L
    from flapjax_b200.flowfields import Constant
    from oracle import uvlm_linear as OL
    from oracle import uvlm_ref as R
    from tests.linear_cpu_ops import OracleOps

    c = cases.wing_heave(m=2, n=2, m_star=m_star, n_steps=1)
    uv = R.UVLMRef([(c.m, c.n, c.m_star)], np.arange(c.n + 1))
    uv.set_design_variables(c.dt, R.Constant(c.u_inf, c.rho), c.zeta_b0, c.hg0)
    st = uv.solve_static()
    want = OL.LinearUVLMRef(uv, st, wake_type, bound_upwash, wake_upwash, unsteady).linearise()
    ref = {k: [a[0] for a in getattr(st, k)] for k in ("zeta_b", "zeta_w", "gamma_b", "gamma_w")}
    cfg = {"wake_type": wake_type, "free_wake": False, "kernel": _lib.FJ_KERNEL_EPSILON, "r_cut": 1e-4,
           "force_r_cut": 1e-4, "dt": c.dt, "rho": c.rho, "flowfield": Constant(c.u_inf, c.rho, True), "t": 0.0,
           "bound_upwash": bound_upwash, "wake_upwash": wake_upwash, "unsteady_force": unsteady}
    lay = L._Layout([(c.m, c.n, c.m_star)], wake_type, bound_upwash, wake_upwash, unsteady)
    rs, ro = L._assemble(OracleOps(None), lay, ref, cfg)
    ns = lay.n_states
    got = {"a": rs[:, :ns], "b": rs[:, ns:], "c": ro[:, :ns], "d": ro[:, ns:]}
    for k in "abcd":
        w = getattr(want, k)
        assert got[k].shape == w.shape, k
        assert np.abs(got[k].numpy() - w).max() <= 1e-8 * max(1.0, np.abs(w).max()), k


@pytest.mark.parametrize("name", LG.PROJECTED)
def test_projections_match_reference(name):
    """Input projection (rigid heave and pitch) and output projection (lift and pitching
    moment) against the reference's own projected linear model; the assembly with the
    oracle's operations, the projections as the product applies them."""
    from flapjax_b200 import linear as L
    from tests.linear_cpu_ops import OracleOps

    g = LG.load(name)
    cfg = LG.config(g, LG.flow_product(g))
    lay = L._Layout(LG.dims(g), cfg["wake_type"], True, True, True)
    rs, ro = L._assemble(OracleOps(None), lay, LG.reference(g), cfg)
    ip, op = LG.projections(g)
    t = lambda x: None if x is None else torch.as_tensor(x)
    jin = tuple(t(j) for j in L._input_jacobians(ip, 3 * lay.NVB))
    fs0 = g["ref_f_steady"].ravel()
    jout = tuple(t(j) for j in L._output_jacobians(op, fs0, np.zeros_like(fs0)))
    ns = lay.n_states
    a, b, c, d = L._project(torch, lay, rs[:, :ns], rs[:, ns:], ro[:, :ns], ro[:, ns:], jin, jout)
    for k, got in zip("abcd", (a, b, c, d)):
        want = g[k]
        assert got.shape == want.shape, k
        assert np.abs(got.numpy() - want).max() <= 1e-8 * max(1.0, np.abs(want).max()), k


def test_projection_argument_checks():
    from flapjax_b200 import linear as L

    ip = L.LinearInputProjection(arg_names=("q",), arg_sizes=(2,), arg_refs=(np.zeros(3),),
                                 to_zeta=lambda q: (np.zeros(6), np.zeros(6)))
    with pytest.raises(ValueError):
        L._input_jacobians(ip, 6)
    ip = L.LinearInputProjection(arg_names=("q",), arg_sizes=(2,), arg_refs=(np.zeros(2),),
                                 to_zeta=lambda q: (np.zeros(5), np.zeros(5)))
    with pytest.raises(ValueError):
        L._input_jacobians(ip, 6)
    jz = np.arange(12.0).reshape(6, 2)
    ip = L.LinearInputProjection(arg_names=("q",), arg_sizes=(2,), arg_refs=(np.zeros(2),),
                                 to_zeta=lambda q: (jz @ q, 2 * jz @ q))
    a, b = L._input_jacobians(ip, 6)
    assert np.allclose(a, jz, atol=1e-8) and np.allclose(b, 2 * jz, atol=1e-8)
    op = L.LinearOutputProjection(name="o", size=1, to_output=lambda fs, fu: np.array([fs.sum() + fu.sum()]))
    jfs, jfu = L._output_jacobians(op, np.ones(6), np.ones(6))
    assert np.allclose(jfs, 1.0) and np.allclose(jfu, 1.0)


def test_layout_follows_reference_slices():
    from flapjax_b200 import linear as L

    lay = L._Layout([(2, 3, 4), (1, 2, 2)], "prescribed", True, False, True)
    nb, nw, nvb, nvw = 6 + 2, 12 + 4, 12 + 6, 20 + 9
    assert [k for k, _ in lay.x_blocks] == ["gamma_b", "gamma_w", "gamma_b_nm1", "zeta_w", "zeta_b"]
    assert lay.x["zeta_w"] == (nb + nw + nb, nb + nw + nb + 3 * nvw)
    assert [k for k, _ in lay.u_blocks] == ["zeta_b", "zeta_b_dot", "nu_b"]
    assert lay.n_inputs == 9 * nvb and lay.n_outputs == 6 * nvb
    frozen = L._Layout([(2, 3, 4)], "frozen", False, False, False)
    assert [k for k, _ in frozen.x_blocks] == ["gamma_b", "gamma_w"]
    assert [k for k, _ in frozen.y_blocks] == ["f_steady"]


def test_diff_lists_follow_compute_jacobians():
    """The differentiated arguments per residual, as the reference's compute_jacobians
    lists them (the golden generator records the reference's own lists)."""
    from flapjax_b200 import linear as L
    from oracle import uvlm_linear as OL

    for wt in ("frozen", "prescribed", "free"):
        for flags in ((True, True, True), (False, True, False), (True, False, True)):
            assert L._diff_lists(wt, *flags) == OL.diff_lists(wt, *flags)
    assert "x:zeta_b" not in L._diff_lists("free", True, True, True)["zeta_w"]
    assert "x:gamma_b" in L._diff_lists("free", True, True, True)["zeta_w"]
    assert "x:gamma_b" not in L._diff_lists("prescribed", True, True, True)["zeta_w"]


def test_linear_system_remove_u_np1_and_argument_checks():
    """LinearSystem.remove_u_np1 (utils/linear.py:714-724) against the oracle's restatement
    on CPU tensors; run's shape checks come before the device march, and run refuses
    matrices that are not on the GPU (the march is fj_lti_march; tests/test_gpu_linear.py
    checks it against the oracle)."""
    from flapjax_b200.linear import LinearSystem
    from oracle.uvlm_linear import LinearSystemRef

    rng = np.random.default_rng(0)
    a = 0.3 * rng.normal(size=(7, 7))
    b, c, d = rng.normal(size=(7, 4)), rng.normal(size=(5, 7)), rng.normal(size=(5, 4))
    u, x0 = rng.normal(size=(9, 4)), rng.normal(size=7)
    t = lambda z: torch.as_tensor(z)
    ours = LinearSystem(t(a), t(b), t(c), t(d), 0.1)
    ref = LinearSystemRef(a, b, c, d, 0.1)
    ours.remove_u_np1()
    ref.remove_u_np1()
    for got, want in ((ours.b, ref.b), (ours.d, ref.d)):
        assert np.allclose(got.numpy(), want, rtol=1e-13, atol=1e-13)
    with pytest.warns(UserWarning):
        ours.remove_u_np1()
    with pytest.raises(RuntimeError, match="CUDA"):
        ours.run(u, x0)
