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

    python tests/golden/make_golden.py

The GPU box has no /root/reference; only the .npz files travel.
"""
from __future__ import annotations

import importlib.abc
import importlib.machinery
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF_SRC = Path("/root/reference/src")


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


if __name__ == "__main__":
    main()
