"""Generate golden vectors by running the REFERENCE's own UVLM source.

FLAPJAX (ben-l-p/flapjax 1.2.1) is pure Python on JAX; JAX is not installed here, so the
reference source under /root/reference/src is executed with ``tests/golden/jaxshim`` (a
NumPy stand-in for the jax API it uses: float64 arrays with ``.at[]`` updates, eager
``vmap``/``lax.map``/``fori_loop``).  The plotting dependency (vtk) is replaced by inert
stub modules and the package ``__init__`` files that pull in the structural solver are
bypassed; every aero module on the path (uvlm.py, aic.py, aero/utils.py, flowfields.py,
data_structures.py, algebra/*) runs unmodified.

Each case is written to ``tests/golden/<name>.npz`` with its inputs and the reference's
time-batched outputs.  Run from the repository root in this container:

    python tests/golden/make_golden.py [case names]

The reference's ``src`` directory defaults to /root/reference/src; set FLAPJAX_REF_SRC to
read it from elsewhere.  The GPU box has no reference checkout; only the .npz files travel.
"""
from __future__ import annotations

import importlib.abc
import importlib.machinery
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF_SRC = Path(os.environ.get("FLAPJAX_REF_SRC", "/root/reference/src"))


class _Stub(types.ModuleType):
    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _Stub(f"{self.__name__}.{name}")

    def __call__(self, *a, **k):
        return _Stub(self.__name__ + "()")


class _StubFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    """Inert modules for the reference's file-output dependencies."""

    PREFIXES = ("vtk", "vtkmodules", "matplotlib", "mpl_toolkits")

    def find_spec(self, name, path, target=None):
        if name.split(".")[0] in self.PREFIXES:
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        m = _Stub(spec.name)
        m.__path__ = []
        return m

    def exec_module(self, module):
        pass


def load_reference():
    sys.path.insert(0, str(HERE / "jaxshim"))
    sys.path.insert(0, str(REF_SRC))
    sys.meta_path.insert(0, _StubFinder())
    src = REF_SRC / "flapjax"
    for pkg, sub in [("flapjax", ""), ("flapjax.aero", "aero"), ("flapjax.structure", "structure"),
                     ("flapjax.coupled", "coupled"), ("flapjax.plotting", "plotting")]:
        m = types.ModuleType(pkg)
        m.__path__ = [str(src / sub) if sub else str(src)]
        sys.modules[pkg] = m
    import jax.numpy as jnp  # the stand-in
    from flapjax.aero import utils as aero_utils
    from flapjax.aero.data_structures import GridDiscretisation
    from flapjax.aero.flowfields import Constant, OneMinusCosine
    from flapjax.aero.uvlm import UVLM

    return types.SimpleNamespace(jnp=jnp, UVLM=UVLM, GridDiscretisation=GridDiscretisation, Constant=Constant,
                                 OneMinusCosine=OneMinusCosine, utils=aero_utils)


FIELDS = ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
          "f_unsteady", "alpha")


def _flow_dict(kind, u_inf, rho, gust=None):
    d = {"flow_kind": kind, "u_inf": np.asarray(u_inf, float), "rho": float(rho)}
    if gust:
        d.update({f"gust_{k}": np.asarray(v, float) for k, v in gust.items()})
    return d


def run_case(ref, name, surfaces, dt, flow, kernel="epsilon", r_cut=None, free_wake=False, mirror=None,
             horseshoe=False, gamma_dot_relaxation=0.7, hg0=None, hg_t=None, hg_dot_t=None, delta_w=None,
             polars=None, polar_circulation_scale=0.0):
    """surfaces: list of (m, n, m_star, zeta_b0, dof_mapping); delta_w: per-surface segment
    lengths (or None entries) of the variable wake discretisation; polars: per-surface
    (n, P, 4) tables of (alpha, cl, cd, cm) (or None entries), handed to the reference as
    jnp.interp callables."""
    if ONLY and name not in ONLY:
        return
    jnp = ref.jnp
    kern = {"epsilon": ref.utils.biot_savart_epsilon, "cutoff": ref.utils.biot_savart_cutoff,
            "plain": ref.utils.biot_savart}[kernel]
    saved_r = ref.utils.R_CUTOFF
    if r_cut is not None:
        ref.utils.R_CUTOFF = r_cut  # module constant read by biot_savart_cutoff (aero/utils.py:648)
    try:
        kw = {}
        if mirror is not None:
            kw = dict(mirror_point=jnp.array(mirror[0]), mirror_normal=jnp.array(mirror[1]))
        if polars is not None:
            def _callable(tab):
                return lambda a: tuple(jnp.interp(a, tab[:, 0], tab[:, q]) for q in (1, 2, 3))

            kw["polars"] = [None if p is None else [_callable(np.asarray(t, float)) for t in p] for p in polars]
            kw["polar_circulation_scale"] = polar_circulation_scale
        uv = ref.UVLM(grid_shapes=[ref.GridDiscretisation(m, n, ms) for m, n, ms, _, _ in surfaces],
                      dof_mapping=[jnp.array(d) for *_, d in surfaces], kernel=kern, free_wake=free_wake,
                      gamma_dot_relaxation=gamma_dot_relaxation, **kw)
        if flow["flow_kind"] == "constant":
            ff = ref.Constant(jnp.array(flow["u_inf"]), flow["rho"], True)
        else:
            ff = ref.OneMinusCosine(jnp.array(flow["u_inf"]), flow["rho"], True,
                                    gust_length=float(flow["gust_length"]),
                                    gust_amplitude=float(flow["gust_amplitude"]))
        dw_arg = None if delta_w is None else [None if d is None else jnp.array(d) for d in delta_w]
        uv.set_design_variables(dt=float(dt), flowfield=ff, zeta_b0=[jnp.array(z) for *_, z, _ in surfaces],
                                hg0=jnp.array(hg0), delta_w=dw_arg)
        st = uv.solve_static(horseshoe=horseshoe)
        out = {"case_name": name, "kernel": kernel, "r_cut": r_cut if r_cut is not None else saved_r,
               "free_wake": free_wake, "horseshoe": horseshoe, "dt": dt, "gamma_dot_relaxation": gamma_dot_relaxation,
               "hg0": hg0, "n_surf": len(surfaces), **flow}
        for i, (m, n, ms, z, d) in enumerate(surfaces):
            if delta_w is not None and delta_w[i] is not None:
                out[f"surf{i}_delta_w"] = np.asarray(delta_w[i], float)
            out[f"surf{i}_dims"] = np.array([m, n, ms])
            out[f"surf{i}_zeta_b0"] = z
            out[f"surf{i}_dof"] = np.asarray(d)
        if polars is not None:
            out["polar_circulation_scale"] = float(polar_circulation_scale)
            for i, p in enumerate(polars):
                if p is not None:
                    out[f"surf{i}_polars"] = np.asarray(p, float)
        if mirror is not None:
            out["mirror_point"] = np.asarray(mirror[0], float)
            out["mirror_normal"] = np.asarray(mirror[1], float)
        for f in FIELDS:
            for i, a in enumerate(getattr(st, f)):
                out[f"static_{f}_{i}"] = np.asarray(a)
        out["static_t"] = np.asarray(st.t)
        if hg_t is not None:
            dy = uv.solve_prescribed_dynamic(init_case=st, hg_t=jnp.array(hg_t), hg_dot_t=jnp.array(hg_dot_t))
            out["hg_t"] = hg_t
            out["hg_dot_t"] = hg_dot_t
            for f in FIELDS:
                for i, a in enumerate(getattr(dy, f)):
                    out[f"dyn_{f}_{i}"] = np.asarray(a)
            out["dyn_t"] = np.asarray(dy.t)
        np.savez_compressed(HERE / f"{name}.npz", **{k: np.asarray(v) for k, v in out.items()})
        print("wrote", name)
    finally:
        ref.utils.R_CUTOFF = saved_r


def run_residual_case(ref, name, c, free_wake=False, kernel="epsilon", r_cut=None, gust=None, slot=2, seed=0):
    """The reference's own UVLM.timestep_residual (aero/uvlm.py:1942-2047) at slot ``slot``
    of a prescribed run, with the states of slot n moved off the solution by seeded noise
    and seeded beam forces.  The beam is not part of this path: a stand-in structure
    object hands the residual the run's node frames for varphi_n / varphi_nm1 (told apart
    by their fill value) and the frame velocities for v_n; the design variables carry no
    overrides and no control surfaces."""
    if ONLY and name not in ONLY:
        return
    jnp = ref.jnp
    from flapjax.algebra.array_utils import ArrayList

    kern = {"epsilon": ref.utils.biot_savart_epsilon, "cutoff": ref.utils.biot_savart_cutoff}[kernel]
    saved_r = ref.utils.R_CUTOFF
    if r_cut is not None:
        ref.utils.R_CUTOFF = r_cut
    try:
        uv = ref.UVLM(grid_shapes=[ref.GridDiscretisation(c.m, c.n, c.m_star)], dof_mapping=[jnp.arange(c.n + 1)],
                      kernel=kern, free_wake=free_wake)
        if gust is None:
            ff = ref.Constant(jnp.array(c.u_inf), c.rho, True)
        else:
            ff = ref.OneMinusCosine(jnp.array(c.u_inf), c.rho, True, gust_length=gust["length"],
                                    gust_amplitude=gust["amplitude"], gust_x0=jnp.array(gust["x0"]))
        uv.set_design_variables(dt=float(c.dt), flowfield=ff, zeta_b0=[jnp.array(c.zeta_b0)], hg0=jnp.array(c.hg0))
        st = uv.solve_static()
        dy = uv.solve_prescribed_dynamic(init_case=st, hg_t=jnp.array(c.hg_t), hg_dot_t=jnp.array(c.hg_dot_t))
        rng = np.random.default_rng(seed)
        keys = ("gamma_b", "gamma_w", "gamma_b_dot", "zeta_w")
        qn = {k: np.asarray(getattr(dy, k)[0][slot]) + 0.01 * rng.normal(size=np.shape(getattr(dy, k)[0][slot]))
              for k in keys}
        qm = {k: np.asarray(getattr(dy, k)[0][slot - 1]) for k in keys}
        n_nodes = c.hg0.shape[0]
        f_beam = rng.normal(size=(n_nodes, 6))
        frames = {1.0: np.asarray(c.hg_t[slot]), 2.0: np.asarray(c.hg_t[slot - 1])}

        class _Beam:
            n_dof = n_nodes * 6

            def case_from_dv(self, dv):
                return self

            def calculate_hg_from_varphi(self, varphi):
                return jnp.array(frames[float(np.asarray(varphi).ravel()[0])])

            def make_hg_dot(self, hg, v):
                return jnp.array(c.hg_dot_t[slot])

        aero_dv = types.SimpleNamespace(flowfield=None, cs_ang_t=None, zeta_b0=None,
                                        get_cs_n=lambda i_ts, dv_full: ({}, {}))
        dv = types.SimpleNamespace(structure=None, aero=aero_dv)
        to_states = lambda q: types.SimpleNamespace(**{k: ArrayList([jnp.array(q[k])]) for k in keys})
        r = uv.timestep_residual(i_ts=slot, varphi_nm1=jnp.full((n_nodes, 6), 2.0),
                                 varphi_n=jnp.full((n_nodes, 6), 1.0), v_n=jnp.zeros((n_nodes, 6)),
                                 t_n=dy.t[slot], q_n=to_states(qn), q_nm1=to_states(qm), dv=dv, dv_full=dv,
                                 f_aero_beam_n=jnp.array(f_beam), struct_obj=_Beam(), approx_grads=False)
        out = {"case_name": name, "kernel": kernel, "r_cut": r_cut if r_cut is not None else saved_r,
               "free_wake": free_wake, "dt": c.dt, "u_inf": c.u_inf, "rho": c.rho, "zeta_b0": c.zeta_b0,
               "hg0": c.hg0, "hg_n": c.hg_t[slot], "hg_dot_n": c.hg_dot_t[slot], "hg_nm1": c.hg_t[slot - 1],
               "t_n": np.asarray(dy.t[slot]), "f_beam_n": f_beam, "dims": np.array([c.m, c.n, c.m_star]),
               "residual": np.asarray(r)}
        if gust is not None:
            out.update(gust_length=gust["length"], gust_amplitude=gust["amplitude"], gust_x0=np.asarray(gust["x0"]))
        for k in keys:
            out[f"q_n_{k}"] = qn[k]
            out[f"q_nm1_{k}"] = qm[k]
        np.savez_compressed(HERE / "residual" / f"{name}.npz", **{k: np.asarray(v) for k, v in out.items()})
        print("wrote residual", name)
    finally:
        ref.utils.R_CUTOFF = saved_r


def run_gradient_case(ref, name, c, free_wake=False, kernel="epsilon", r_cut=None, gust=None, delta_w=None,
                      mirror=None, n_dir=2, h=1e-6, seed=0):
    """Directional derivatives of the reference's own forward: J(zeta_b0) = time-mean CL over
    steps 1..N (sum_n fw_n . F_n, F_n the total vertex force of UVLM.solve_prescribed_dynamic
    from the static solve), and (J(z + h d) - J(z - h d)) / 2h for ``n_dir`` seeded unit-scale
    directions d.  With h = 1e-6 in float64 the truncation error is O(h^2) and the rounding
    error about 1e-16 |J| / h, both far below the 1e-6 the adjoint is held to."""
    if ONLY and name not in ONLY:
        return
    jnp = ref.jnp
    kern = {"epsilon": ref.utils.biot_savart_epsilon, "cutoff": ref.utils.biot_savart_cutoff}[kernel]
    saved_r = ref.utils.R_CUTOFF
    if r_cut is not None:
        ref.utils.R_CUTOFF = r_cut
    a = np.deg2rad(c.alpha_deg)
    e_l = np.array((-np.sin(a), 0.0, np.cos(a)))
    q = 0.5 * c.rho * c.u_mag ** 2 * c.s_ref

    def objective(z0):
        kw = {} if mirror is None else dict(mirror_point=jnp.array(mirror[0]), mirror_normal=jnp.array(mirror[1]))
        uv = ref.UVLM(grid_shapes=[ref.GridDiscretisation(c.m, c.n, c.m_star)], dof_mapping=[jnp.arange(c.n + 1)],
                      kernel=kern, free_wake=free_wake, **kw)
        ff = (ref.Constant(jnp.array(c.u_inf), c.rho, True) if gust is None else
              ref.OneMinusCosine(jnp.array(c.u_inf), c.rho, True, gust_length=gust["length"],
                                 gust_amplitude=gust["amplitude"], gust_x0=jnp.array(gust["x0"])))
        uv.set_design_variables(dt=float(c.dt), flowfield=ff, zeta_b0=[jnp.array(z0)], hg0=jnp.array(c.hg0),
                                delta_w=None if delta_w is None else [jnp.array(delta_w)])
        dy = uv.solve_prescribed_dynamic(init_case=uv.solve_static(), hg_t=jnp.array(c.hg_t),
                                         hg_dot_t=jnp.array(c.hg_dot_t))
        ft = np.asarray(dy.f_steady[0]).sum(axis=(1, 2)) + np.asarray(dy.f_unsteady[0]).sum(axis=(1, 2))
        return float(np.sum(ft[1:] @ e_l) / (q * c.n_steps))

    try:
        z0 = np.asarray(c.zeta_b0, float)
        rng = np.random.default_rng(seed)
        dirs = rng.normal(size=(n_dir,) + z0.shape) * 0.1
        J = objective(z0)
        dJ = np.array([(objective(z0 + h * d) - objective(z0 - h * d)) / (2 * h) for d in dirs])
        out = {"case_name": name, "kernel": kernel, "r_cut": r_cut if r_cut is not None else saved_r,
               "free_wake": free_wake, "J": J, "dJ": dJ, "directions": dirs, "h": h}
        if gust is not None:
            out.update(gust_length=gust["length"], gust_amplitude=gust["amplitude"], gust_x0=np.asarray(gust["x0"]))
        if delta_w is not None:
            out["delta_w"] = np.asarray(delta_w, float)
        if mirror is not None:
            out["mirror_point"] = np.asarray(mirror[0], float)
            out["mirror_normal"] = np.asarray(mirror[1], float)
        np.savez_compressed(HERE / "gradient" / f"{name}.npz", **{k: np.asarray(v) for k, v in out.items()})
        print("wrote gradient", name, J, dJ)
    finally:
        ref.utils.R_CUTOFF = saved_r


def run_linear_case(ref, name, c, wake_type, free_wake=False, kernel="epsilon", r_cut=None, gust=None, mirror=None,
                    n_run=6, h=1e-6, seed=0, delta_w=None):
    """The reference's own linearised UVLM (aero/linear/linear_uvlm.py) about the static
    solution of case ``c``.  ``LinearUVLM.compute_jacobians`` supplies, per residual, the
    step function, its arguments and the arguments it differentiates; jax.jacrev is
    replaced by central differences of those same step functions (h = 1e-6 in float64:
    truncation O(h^2), rounding about 1e-16 / h), and the blocks are assembled into A, B,
    C, D by the reference's ``construct_named_block_jacobian`` in ``linearise``'s order.
    The reference's ``LinearSystem.run`` then marches those matrices over ``n_run`` seeded
    input perturbations.  Also stored: the step's packed outputs at the reference point
    and at one seeded perturbation of every input and state.

    With a variable wake (``delta_w``) the linear model's step holds the wake's arc lengths
    with jax.lax.stop_gradient (``linearise_variable_wake``, aero/utils.py:465-468), so
    jacrev differentiates with the arc lengths fixed at the reference point.  The stand-in's
    stop_gradient is the identity; here it records the arc lengths of the reference-point
    step and hands those back to every differenced step, which is what jacrev sees."""
    if ONLY and name not in ONLY:
        return
    jnp = ref.jnp
    from flapjax.aero.linear.linear_uvlm import LinearUVLM
    from flapjax.algebra.array_utils import construct_named_block_jacobian
    from flapjax.utils.linear import LinearSystem

    kern = {"epsilon": ref.utils.biot_savart_epsilon, "cutoff": ref.utils.biot_savart_cutoff}[kernel]
    saved_r = ref.utils.R_CUTOFF
    if r_cut is not None:
        ref.utils.R_CUTOFF = r_cut
    try:
        kw = {} if mirror is None else dict(mirror_point=jnp.array(mirror[0]), mirror_normal=jnp.array(mirror[1]))
        uv = ref.UVLM(grid_shapes=[ref.GridDiscretisation(c.m, c.n, c.m_star)], dof_mapping=[jnp.arange(c.n + 1)],
                      kernel=kern, free_wake=free_wake, **kw)
        ff = (ref.Constant(jnp.array(c.u_inf), c.rho, True) if gust is None else
              ref.OneMinusCosine(jnp.array(c.u_inf), c.rho, True, gust_length=gust["length"],
                                 gust_amplitude=gust["amplitude"], gust_x0=jnp.array(gust["x0"])))
        uv.set_design_variables(dt=float(c.dt), flowfield=ff, zeta_b0=[jnp.array(c.zeta_b0)], hg0=jnp.array(c.hg0),
                                delta_w=None if delta_w is None else [jnp.array(delta_w)])
        st = uv.solve_static()
        lin = LinearUVLM(uv, st, wake_type=wake_type, skip_linearisation=True)
        residuals = lin.compute_jacobians()
        import jax.lax as shim_lax

        held = {"mode": "off", "vals": [], "k": 0}

        def held_stop_gradient(x):
            if held["mode"] == "record":
                held["vals"].append(np.array(x))
                return x
            if held["mode"] == "replay":
                v = held["vals"][held["k"]]
                held["k"] += 1
                return jnp.array(v)
            return x

        shim_lax.stop_gradient = held_stop_gradient

        def full_step(mode="replay", **kwargs):
            held["mode"], held["k"] = mode, 0
            x1, y0 = lin._step_from_vecs(**kwargs)
            return np.asarray(lin.pack_state_vector(x1)), np.asarray(lin.pack_output_vector(y0))

        # every differentiated argument, each perturbed once per column and sign; all
        # other arguments stay at the reference, as in the residual functions' defaults
        ref_args = {}
        for _, args, diff in residuals.values():
            for k in diff:
                ref_args[k] = np.asarray(args[k], float)
        x_ref, y_ref = full_step(mode="record")
        cols = {}
        for k, v in ref_args.items():
            jx = np.zeros((x_ref.size, v.size))
            jy = np.zeros((y_ref.size, v.size))
            for j in range(v.size):
                vp, vm = v.copy(), v.copy()
                vp[j] += h
                vm[j] -= h
                xp, yp = full_step(**{k: jnp.array(vp)})
                xm, ym = full_step(**{k: jnp.array(vm)})
                jx[:, j] = (xp - xm) / (2 * h)
                jy[:, j] = (yp - ym) / (2 * h)
            cols[k] = (jx, jy)
            print(" ", name, k, v.size)

        def rows(slices, nm):
            comp = slices[nm]
            sl = comp.slices if isinstance(comp.slices, slice) else comp.slices[0]
            return sl

        jac = {}
        for res, (_, _, diff) in residuals.items():
            is_out = res in ("f_steady", "f_unsteady")
            sl = rows(lin.output_slices if is_out else lin.state_slices, res)
            jac[res] = {k: jnp.array(cols[k][1 if is_out else 0][sl]) for k in diff}
        state_specs = [("gamma_b", "gamma_b_n_vec"), ("gamma_w", "gamma_w_n_vec"), ("gamma_b_nm1", "gamma_b_nm1_vec"),
                       ("zeta_w", "zeta_w_n_vec"), ("zeta_b", "zeta_b_n_vec")]
        state_specs = [(a, b) for a, b in state_specs if lin.state_slices[a].enabled]
        sizes = {"gamma_b": st.gamma_b.size, "gamma_w": st.gamma_w.size, "gamma_b_nm1": st.gamma_b.size,
                 "zeta_w": st.zeta_w.size, "zeta_b": st.zeta_b.size}
        input_specs = [("zeta_b_np1_vec", st.zeta_b.size), ("zeta_b_dot_np1_vec", st.zeta_b.size),
                       ("nu_b_np1_vec", st.zeta_b.size), ("nu_w_np1_vec", st.zeta_w.size)]
        output_specs = [("f_steady", st.zeta_b.size * 1), ("f_unsteady", st.zeta_b.size)]
        s_names = [a for a, _ in state_specs]
        s_keys = [b for _, b in state_specs]
        s_sizes = [sizes[a] for a in s_names]
        a_ = construct_named_block_jacobian(tuple(jac[k] for k in s_names), s_keys, s_sizes, s_sizes)
        b_ = construct_named_block_jacobian(tuple(jac[k] for k in s_names), [k for k, _ in input_specs],
                                            [v for _, v in input_specs], s_sizes)
        c_ = construct_named_block_jacobian(tuple(jac[k] for k, _ in output_specs), s_keys, s_sizes,
                                            [v for _, v in output_specs])
        d_ = construct_named_block_jacobian(tuple(jac[k] for k, _ in output_specs), [k for k, _ in input_specs],
                                            [v for _, v in input_specs], [v for _, v in output_specs])
        sys_ = LinearSystem(a=a_, b=b_, c=c_, d=d_, dt=float(c.dt))
        rng = np.random.default_rng(seed)
        u_run = 1e-3 * rng.normal(size=(n_run, lin.n_inputs))
        x0 = 1e-3 * rng.normal(size=lin.n_states)
        x_run, y_run = sys_.run(jnp.array(u_run), jnp.array(x0))
        # the nonlinear step at one seeded perturbation of every argument
        pert = {k: v + 1e-3 * rng.normal(size=v.shape) for k, v in ref_args.items()}
        x_p, y_p = full_step(mode="off", **{k: jnp.array(v) for k, v in pert.items()})
        out = {"case_name": name, "wake_type": wake_type, "kernel": kernel,
               "r_cut": r_cut if r_cut is not None else saved_r, "free_wake": free_wake, "dt": c.dt,
               "u_inf": c.u_inf, "rho": c.rho, "zeta_b0": c.zeta_b0, "hg0": c.hg0,
               "dims": np.array([c.m, c.n, c.m_star]), "h": h,
               "a": np.asarray(a_), "b": np.asarray(b_), "c": np.asarray(c_), "d": np.asarray(d_),
               "u_run": u_run, "x0_run": x0, "x_run": np.asarray(x_run), "y_run": np.asarray(y_run),
               "x_ref": x_ref, "y_ref": y_ref, "x_pert": x_p, "y_pert": y_p}
        for k, v in pert.items():
            out[f"pert_{k}"] = v
        for f in ("zeta_b", "zeta_w", "gamma_b", "gamma_w", "f_steady"):
            out[f"ref_{f}"] = np.asarray(getattr(st, f)[0])
        if gust is not None:
            out.update(gust_length=gust["length"], gust_amplitude=gust["amplitude"], gust_x0=np.asarray(gust["x0"]))
        if mirror is not None:
            out["mirror_point"] = np.asarray(mirror[0], float)
            out["mirror_normal"] = np.asarray(mirror[1], float)
        if delta_w is not None:
            out["delta_w"] = np.asarray(delta_w, float)
        np.savez_compressed(HERE / "linear" / f"{name}.npz", **{k: np.asarray(v) for k, v in out.items()})
        print("wrote linear", name)
    finally:
        ref.utils.R_CUTOFF = saved_r
        import jax.lax as shim_lax

        shim_lax.stop_gradient = lambda x: x


def run_linear_projected_case(ref, name, c, wake_type, ea_x=0.0, h=1e-6, seed=0):
    """The reference's linear model with an input projection (rigid heave and pitch) and an
    output projection (lift and pitching moment): compute_jacobians(input_projection=,
    output_projection=) supplies the projected residual functions and their arguments;
    central differences of those functions (h = 1e-6) in place of jacrev, assembled as
    linearise does with projections (aero/linear/linear_uvlm.py:727-829)."""
    if ONLY and name not in ONLY:
        return
    jnp = ref.jnp
    from flapjax.aero.linear.linear_uvlm import LinearInputProjection, LinearOutputProjection, LinearUVLM
    from flapjax.algebra.array_utils import construct_named_block_jacobian

    uv = ref.UVLM(grid_shapes=[ref.GridDiscretisation(c.m, c.n, c.m_star)], dof_mapping=[jnp.arange(c.n + 1)],
                  kernel=ref.utils.biot_savart_epsilon)
    uv.set_design_variables(dt=float(c.dt), flowfield=ref.Constant(jnp.array(c.u_inf), c.rho, True),
                            zeta_b0=[jnp.array(c.zeta_b0)], hg0=jnp.array(c.hg0))
    st = uv.solve_static()
    lin = LinearUVLM(uv, st, wake_type=wake_type, skip_linearisation=True)
    from tests.linear_golden import rigid_projections

    names, sizes, to_zeta, out_size, to_output = rigid_projections(jnp, np.asarray(st.zeta_b[0]), ea_x)
    refs = (jnp.zeros(2), jnp.zeros(2))
    ip = LinearInputProjection(arg_names=names, arg_sizes=sizes, arg_refs=refs, to_zeta=to_zeta)
    op = LinearOutputProjection(name="lift_moment", size=out_size, to_output=to_output)
    residuals = lin.compute_jacobians(input_projection=ip, output_projection=op)
    jac = {}
    for res, (func, args, diff) in residuals.items():
        f0 = np.asarray(func(**args)).ravel()
        jac[res] = {}
        for k in diff:
            v = np.asarray(args[k], float)
            blk = np.zeros((f0.size, v.size))
            for j in range(v.size):
                vp, vm = v.copy(), v.copy()
                vp[j] += h
                vm[j] -= h
                fp = np.asarray(func(**{**args, k: jnp.array(vp)})).ravel()
                fm = np.asarray(func(**{**args, k: jnp.array(vm)})).ravel()
                blk[:, j] = (fp - fm) / (2 * h)
            jac[res][k] = jnp.array(blk)
        print(" ", name, res, diff)
    state_specs = [("gamma_b", "gamma_b_n_vec"), ("gamma_w", "gamma_w_n_vec"), ("gamma_b_nm1", "gamma_b_nm1_vec"),
                   ("zeta_w", "zeta_w_n_vec"), ("zeta_b", "zeta_b_n_vec")]
    state_specs = [(a, b) for a, b in state_specs if lin.state_slices[a].enabled]
    sizes_s = {"gamma_b": st.gamma_b.size, "gamma_w": st.gamma_w.size, "gamma_b_nm1": st.gamma_b.size,
               "zeta_w": st.zeta_w.size, "zeta_b": st.zeta_b.size}
    input_specs = list(zip(names, sizes)) + [("nu_b_np1_vec", st.zeta_b.size), ("nu_w_np1_vec", st.zeta_w.size)]
    s_names = [a for a, _ in state_specs]
    s_keys = [b for _, b in state_specs]
    s_sz = [sizes_s[a] for a in s_names]
    a_ = construct_named_block_jacobian(tuple(jac[k] for k in s_names), s_keys, s_sz, s_sz)
    b_ = construct_named_block_jacobian(tuple(jac[k] for k in s_names), [k for k, _ in input_specs],
                                        [v for _, v in input_specs], s_sz)
    c_ = construct_named_block_jacobian((jac["lift_moment"],), s_keys, s_sz, [out_size])
    d_ = construct_named_block_jacobian((jac["lift_moment"],), [k for k, _ in input_specs],
                                        [v for _, v in input_specs], [out_size])
    out = {"case_name": name, "wake_type": wake_type, "kernel": "epsilon", "r_cut": ref.utils.R_CUTOFF,
           "free_wake": False, "dt": c.dt, "u_inf": c.u_inf, "rho": c.rho, "zeta_b0": c.zeta_b0, "hg0": c.hg0,
           "dims": np.array([c.m, c.n, c.m_star]), "h": h, "ea_x": ea_x,
           "a": np.asarray(a_), "b": np.asarray(b_), "c": np.asarray(c_), "d": np.asarray(d_)}
    for f in ("zeta_b", "zeta_w", "gamma_b", "gamma_w", "f_steady"):
        out[f"ref_{f}"] = np.asarray(getattr(st, f)[0])
    np.savez_compressed(HERE / "linear" / f"{name}.npz", **{k: np.asarray(v) for k, v in out.items()})
    print("wrote linear", name)


def run_fsi_case(ref, name, c, free_wake=False, kernel="epsilon", r_cut=None, n_iter=3):
    """A fluid-structure loop with the shape of the reference's fsi_convergence_loop
    (structure/beam.py:2612-2697): the reference's own UVLM.case_solve, then the solved
    slot's AeroCase.project_forcing_to_beam, then a structural update, ``n_iter`` times per
    step (tests/fsi_standin.py, a typical-section stand-in for the beam).  Stored per call:
    the frames, their rates and the projected loads; at the end the case's slots, the
    structural history, and the reference's get_states / gamma_full / zeta_full of one slot
    and its projection with and without the unsteady forces."""
    if ONLY and name not in ONLY:
        return
    jnp = ref.jnp
    from flapjax.aero.data_structures import AeroCase as RefAeroCase

    from tests.fsi_standin import TypicalSection, run_fsi

    kern = {"epsilon": ref.utils.biot_savart_epsilon, "cutoff": ref.utils.biot_savart_cutoff}[kernel]
    saved_r = ref.utils.R_CUTOFF
    if r_cut is not None:
        ref.utils.R_CUTOFF = r_cut
    try:
        uv = ref.UVLM(grid_shapes=[ref.GridDiscretisation(c.m, c.n, c.m_star)], dof_mapping=[jnp.arange(c.n + 1)],
                      kernel=kern, free_wake=free_wake)
        uv.set_design_variables(dt=float(c.dt), flowfield=ref.Constant(jnp.array(c.u_inf), c.rho, True),
                                zeta_b0=[jnp.array(c.zeta_b0)], hg0=jnp.array(c.hg0))
        st = uv.solve_static()
        case = RefAeroCase.initialise(st, c.n_tstep)
        struct = TypicalSection(c.hg0[:, 1, 3])
        rec = []
        case, (x, v, a) = run_fsi(uv, struct, case, c.n_tstep, c.dt, n_iter=n_iter, record=rec)
        out = {"case_name": name, "kernel": kernel, "r_cut": r_cut if r_cut is not None else saved_r,
               "free_wake": free_wake, "dt": c.dt, "u_inf": c.u_inf, "rho": c.rho, "zeta_b0": c.zeta_b0,
               "hg0": c.hg0, "dims": np.array([c.m, c.n, c.m_star]), "n_tstep": c.n_tstep, "n_iter": n_iter,
               "rec_i": np.array([r[0] for r in rec]), "rec_it": np.array([r[1] for r in rec]),
               "rec_hg": np.stack([r[2] for r in rec]), "rec_hg_dot": np.stack([r[3] for r in rec]),
               "rec_f": np.stack([r[4] for r in rec]), "x": x, "v": v, "a": a}
        for f in FIELDS:
            out[f"dyn_{f}"] = np.asarray(getattr(case, f)[0])
        out["dyn_t"] = np.asarray(case.t)
        slot = c.n_tstep - 1
        out["states_slot"] = slot
        out["states_ravel"] = np.asarray(case.get_states(slot).ravel())
        out["gamma_full"] = np.concatenate([np.ravel(g) for g in case.gamma_full(slot)])
        out["zeta_full"] = np.concatenate([np.ravel(z) for z in case.zeta_full(slot)])
        rng = np.random.default_rng(11)
        th = rng.normal(size=(c.n + 1, 3)) * 0.2
        rmat = np.stack([_rot(t) for t in th])
        out["proj_rmat"] = rmat
        out["proj_unsteady"] = np.asarray(case.project_forcing_to_beam(slot, jnp.array(rmat), uv.zeta_b0, True))
        out["proj_steady"] = np.asarray(case.project_forcing_to_beam(slot, jnp.array(rmat), uv.zeta_b0, False))
        np.savez_compressed(HERE / "fsi" / f"{name}.npz", **{k: np.asarray(v_) for k, v_ in out.items()})
        print("wrote fsi", name, len(rec), "calls")
    finally:
        ref.utils.R_CUTOFF = saved_r


def _rot(t):
    """Rotation matrix of the rotation vector t (Rodrigues)."""
    a = float(np.linalg.norm(t))
    k = t / a
    kx = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
    return np.eye(3) + np.sin(a) * kx + (1.0 - np.cos(a)) * kx @ kx


ONLY: set[str] = set()


def main():
    ONLY.update(sys.argv[1:])  # optional case names: regenerate only those
    sys.path.insert(0, str(ROOT))
    from flapjax_b200 import cases

    ref = load_reference()

    c = cases.wing_heave(m=3, n=4, m_star=5, n_steps=4)
    run_case(ref, "heave_epsilon", [(c.m, c.n, c.m_star, c.zeta_b0, np.arange(c.n + 1))], c.dt,
             _flow_dict("constant", c.u_inf, c.rho), hg0=c.hg0, hg_t=c.hg_t, hg_dot_t=c.hg_dot_t)

    c = cases.wing_free(m=3, n=5, m_star=6, n_steps=4)
    run_case(ref, "free_cutoff_1e-3", [(c.m, c.n, c.m_star, c.zeta_b0, np.arange(c.n + 1))], c.dt,
             _flow_dict("constant", c.u_inf, c.rho), kernel="cutoff", r_cut=1e-3, free_wake=True,
             hg0=c.hg0, hg_t=c.hg_t, hg_dot_t=c.hg_dot_t)

    c = cases.wing_free(m=2, n=4, m_star=4, n_steps=3)
    run_case(ref, "free_epsilon", [(c.m, c.n, c.m_star, c.zeta_b0, np.arange(c.n + 1))], c.dt,
             _flow_dict("constant", c.u_inf, c.rho), free_wake=True, hg0=c.hg0, hg_t=c.hg_t, hg_dot_t=c.hg_dot_t)

    c = cases.wing_heave(m=3, n=4, m_star=4, n_steps=3)
    run_case(ref, "mirror_heave", [(c.m, c.n, c.m_star, c.zeta_b0, np.arange(c.n + 1))], c.dt,
             _flow_dict("constant", c.u_inf, c.rho), mirror=(np.zeros(3), np.array([0.0, 1.0, 0.0])),
             hg0=c.hg0, hg_t=c.hg_t, hg_dot_t=c.hg_dot_t)

    c = cases.wing_heave(m=3, n=5, m_star=6, n_steps=1)
    run_case(ref, "horseshoe_static", [(c.m, c.n, c.m_star, c.zeta_b0, np.arange(c.n + 1))], c.dt,
             _flow_dict("constant", c.u_inf, c.rho), horseshoe=True, hg0=c.hg0)

    c = cases.wing_pitch(m=3, n=4, m_star=5, n_steps=4, n_ctrl=3)
    run_case(ref, "pitch_twist", [(c.m, c.n, c.m_star, c.zeta_b0, np.arange(c.n + 1))], c.dt,
             _flow_dict("constant", c.u_inf, c.rho), hg0=c.hg0, hg_t=c.hg_t, hg_dot_t=c.hg_dot_t)

    # gust: the 1-cos gust enters the wing during the run (gust_length = half length)
    c = cases.wing_heave(m=3, n=4, m_star=5, n_steps=6)
    run_case(ref, "gust_heave", [(c.m, c.n, c.m_star, c.zeta_b0, np.arange(c.n + 1))], c.dt,
             _flow_dict("gust", c.u_inf, c.rho, {"length": 0.6, "amplitude": 0.05}), hg0=c.hg0, hg_t=c.hg_t,
             hg_dot_t=c.hg_dot_t)

    # two surfaces: a wing and a tail on separate node sets
    wing = cases.wing_heave(m=3, n=4, m_star=4, n_steps=3)
    tail = np.zeros((3, 3, 3))
    tail[..., 0] = (np.linspace(0.0, 0.5, 3) - 0.125)[:, None] + 3.0
    tail[..., 2] = 0.2
    hg_tail = np.zeros((3, 4, 4))
    hg_tail[:, :3, :3] = np.eye(3)
    hg_tail[:, 1, 3] = np.linspace(0.0, 1.5, 3)
    hg_tail[:, 3, 3] = 1.0
    hg0 = np.concatenate([wing.hg0, hg_tail])
    hg_t = np.concatenate([wing.hg_t, np.repeat(hg_tail[None], wing.hg_t.shape[0], 0)], axis=1)
    hg_dot_t = np.concatenate([wing.hg_dot_t, np.zeros((wing.hg_t.shape[0], 3, 4, 4))], axis=1)
    run_case(ref, "two_surfaces", [(3, 4, 4, wing.zeta_b0, np.arange(5)), (2, 2, 3, tail, np.arange(5, 8))],
             wing.dt, _flow_dict("constant", wing.u_inf, wing.rho), hg0=hg0, hg_t=hg_t, hg_dot_t=hg_dot_t)

    # variable wake discretisation (delta_w): segments growing by 15 % per row, prescribed
    # heave and free wake
    c = cases.wing_heave(m=3, n=4, m_star=6, n_steps=5)
    dw = c.dt * c.u_mag * 1.15 ** np.arange(c.m_star)
    run_case(ref, "variable_wake_heave", [(c.m, c.n, c.m_star, c.zeta_b0, np.arange(c.n + 1))], c.dt,
             _flow_dict("constant", c.u_inf, c.rho), hg0=c.hg0, hg_t=c.hg_t, hg_dot_t=c.hg_dot_t, delta_w=[dw])
    # polar correction (aero/utils.py:276-397): per-strip tables, circulation blend 0.5
    c = cases.wing_heave(m=3, n=4, m_star=4, n_steps=3)
    rng = np.random.default_rng(5)
    tabs = []
    for _ in range(c.n):
        al = np.sort(rng.uniform(-0.2, 0.3, 7))
        tabs.append(np.stack([al, 5.5 * al + rng.normal(0, 0.05, 7), 0.01 + 0.3 * al ** 2,
                              -0.04 + 0.02 * rng.normal(size=7)], axis=1))
    run_case(ref, "polar_heave", [(c.m, c.n, c.m_star, c.zeta_b0, np.arange(c.n + 1))], c.dt,
             _flow_dict("constant", c.u_inf, c.rho), hg0=c.hg0, hg_t=c.hg_t, hg_dot_t=c.hg_dot_t,
             polars=[np.stack(tabs)], polar_circulation_scale=0.5)

    c = cases.wing_free(m=2, n=4, m_star=5, n_steps=4)
    dw = c.dt * c.u_mag * 1.2 ** np.arange(c.m_star)
    run_case(ref, "variable_wake_free", [(c.m, c.n, c.m_star, c.zeta_b0, np.arange(c.n + 1))], c.dt,
             _flow_dict("constant", c.u_inf, c.rho), free_wake=True, hg0=c.hg0, hg_t=c.hg_t, hg_dot_t=c.hg_dot_t,
             delta_w=[dw])


    # the time-step residual of the coupled adjoint (aero side)
    (HERE / "residual").mkdir(exist_ok=True)
    c = cases.wing_heave(m=3, n=4, m_star=4, n_steps=3)
    run_residual_case(ref, "residual_heave", c)
    c = cases.wing_free(m=3, n=4, m_star=4, n_steps=3, seed=1)
    run_residual_case(ref, "residual_free_cutoff", c, free_wake=True, kernel="cutoff", r_cut=1e-3)
    run_residual_case(ref, "residual_free_gust", c, free_wake=True, kernel="cutoff", r_cut=1e-3,
                      gust={"length": 2.0, "amplitude": 0.1, "x0": [-3.0, 0.0, 0.0]})


    # directional derivatives of the reference's own forward, for the adjoint
    (HERE / "gradient").mkdir(exist_ok=True)
    run_gradient_case(ref, "gradient_pitch", cases.wing_pitch(m=3, n=4, m_star=4, n_steps=4, n_ctrl=3, seed=3))
    c = cases.wing_free(m=3, n=4, m_star=4, n_steps=3, seed=1)
    run_gradient_case(ref, "gradient_free_cutoff", c, free_wake=True, kernel="cutoff", r_cut=1e-3)
    run_gradient_case(ref, "gradient_free_gust", c, free_wake=True, kernel="cutoff", r_cut=1e-3,
                      gust={"length": 2.0, "amplitude": 0.1, "x0": [-3.0, 0.0, 0.0]})
    c = cases.wing_pitch(m=3, n=4, m_star=5, n_steps=4, n_ctrl=3, seed=3)
    run_gradient_case(ref, "gradient_pitch_delta_w", c, delta_w=c.dt * c.u_mag * 1.2 ** np.arange(c.m_star))
    c = cases.wing_free(m=3, n=4, m_star=4, n_steps=3, seed=1)
    run_gradient_case(ref, "gradient_free_mirror", c, free_wake=True, kernel="cutoff", r_cut=1e-3,
                      mirror=([0.0, 0.0, 0.0], [0.0, 1.0, 0.0]))

    # the linearised UVLM about a static solution: A, B, C, D by central differences of the
    # reference's own step functions, and its LinearSystem.run
    (HERE / "linear").mkdir(exist_ok=True)
    run_linear_case(ref, "linear_frozen", cases.wing_heave(m=2, n=3, m_star=3, n_steps=1), "frozen")
    c = cases.wing_free(m=2, n=3, m_star=3, n_steps=1, seed=2)
    run_linear_case(ref, "linear_free_gust_mirror", c, "free", free_wake=True, kernel="cutoff", r_cut=1e-3,
                    gust={"length": 2.0, "amplitude": 0.1, "x0": [-1.5, 0.0, 0.0]},
                    mirror=([0.0, -0.5, 0.0], [0.0, 1.0, 0.0]))
    c = cases.wing_pitch(m=2, n=3, m_star=3, n_steps=1, n_ctrl=3, seed=4)
    run_linear_case(ref, "linear_prescribed", c, "prescribed")
    c = cases.wing_heave(m=2, n=3, m_star=3, n_steps=1)
    run_linear_case(ref, "linear_delta_w_frozen", c, "frozen", delta_w=c.dt * c.u_mag * 1.2 ** np.arange(c.m_star))
    c = cases.wing_free(m=2, n=3, m_star=3, n_steps=1, seed=5)
    run_linear_case(ref, "linear_delta_w_free", c, "free", free_wake=True, kernel="cutoff", r_cut=1e-3,
                    delta_w=c.dt * c.u_mag * 1.15 ** np.arange(c.m_star))
    c = cases.wing_heave(m=2, n=3, m_star=3, n_steps=1)
    run_linear_projected_case(ref, "linear_projected_frozen", c, "frozen")
    run_linear_projected_case(ref, "linear_projected_prescribed", c, "prescribed", ea_x=0.1)

    # fluid-structure loops: the reference's case_solve + project_forcing_to_beam driven by
    # a typical-section stand-in for the beam (prescribed and free wake)
    (HERE / "fsi").mkdir(exist_ok=True)
    run_fsi_case(ref, "fsi_heave", cases.wing_heave(m=3, n=6, m_star=6, n_steps=6))
    run_fsi_case(ref, "fsi_free_cutoff", cases.wing_free(m=3, n=6, m_star=5, n_steps=5, seed=2), free_wake=True,
                 kernel="cutoff", r_cut=1e-3)


if __name__ == "__main__":
    main()
