"""Loading of the linear-model golden cases (tests/golden/linear/*.npz, written by
tests/golden/make_golden.py from the reference's own LinearUVLM)."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "linear"
CASES = ("linear_frozen", "linear_free_gust_mirror", "linear_prescribed")
PROJECTED = ("linear_projected_frozen", "linear_projected_prescribed")
VARIABLE = ("linear_delta_w_frozen", "linear_delta_w_free")


def load(name):
    return dict(np.load(GOLDEN / f"{name}.npz", allow_pickle=False))


def mirror_of(g):
    return None if "mirror_point" not in g else (g["mirror_point"], g["mirror_normal"])


def flow_oracle(g):
    from oracle import uvlm_ref as R

    if "gust_length" in g:
        return R.OneMinusCosine(g["u_inf"], float(g["rho"]), True, float(g["gust_length"]),
                                float(g["gust_amplitude"]), gust_x0=g["gust_x0"])
    return R.Constant(g["u_inf"], float(g["rho"]))


def flow_product(g):
    from flapjax_b200 import Constant, OneMinusCosine

    if "gust_length" in g:
        return OneMinusCosine(g["u_inf"], float(g["rho"]), True, gust_length=float(g["gust_length"]),
                              gust_amplitude=float(g["gust_amplitude"]), gust_x0=g["gust_x0"])
    return Constant(g["u_inf"], float(g["rho"]), True)


def kernel_id(g):
    from flapjax_b200 import _lib

    return {"epsilon": _lib.FJ_KERNEL_EPSILON, "cutoff": _lib.FJ_KERNEL_CUTOFF}[str(g["kernel"])]


def config(g, flowfield):
    from flapjax_b200 import _lib

    kid = kernel_id(g)
    return {"wake_type": str(g["wake_type"]), "free_wake": bool(g["free_wake"]), "kernel": kid,
            "r_cut": float(g["r_cut"]), "force_r_cut": float(g["r_cut"]) if kid == _lib.FJ_KERNEL_CUTOFF else 1e-4,
            "dt": float(g["dt"]), "rho": float(g["rho"]), "flowfield": flowfield, "t": 0.0, "bound_upwash": True,
            "wake_upwash": True, "unsteady_force": True, "delta_w": [g["delta_w"]] if "delta_w" in g else None}


def reference(g):
    return {"zeta_b": [g["ref_zeta_b"]], "zeta_w": [g["ref_zeta_w"]], "gamma_b": [g["ref_gamma_b"]],
            "gamma_w": [g["ref_gamma_w"]]}


def dims(g):
    m, n, w = (int(v) for v in g["dims"])
    return [(m, n, w)]


def two_surfaces():
    """A wing (2 x 3, 3 wake rows) and a tail (2 x 2, 2 wake rows) on separate node sets:
    (dims, zeta_b0 per surface, dof mappings, hg0, wing case)."""
    from flapjax_b200 import cases

    wing = cases.wing_heave(m=2, n=3, m_star=3, n_steps=1)
    tail = np.zeros((3, 3, 3))
    tail[..., 0] = (np.linspace(0.0, 0.5, 3) - 0.125)[:, None] + 3.0
    tail[..., 2] = 0.2
    hg_tail = np.zeros((3, 4, 4))
    hg_tail[:, :3, :3] = np.eye(3)
    hg_tail[:, 1, 3] = np.linspace(0.0, 1.5, 3)
    hg_tail[:, 3, 3] = 1.0
    hg0 = np.concatenate([wing.hg0, hg_tail])
    return [(2, 3, 3), (2, 2, 2)], [wing.zeta_b0, tail], [np.arange(4), np.arange(4, 7)], hg0, wing


def two_surface_oracle(wake_type, free, kernel, r_cut=1e-3):
    from oracle import uvlm_linear as OL
    from oracle import uvlm_ref as R

    dims, z0, dofs, hg0, wing = two_surfaces()
    uv = R.UVLMRef(dims, dofs, kernel=kernel, r_cut=r_cut, free_wake=free)
    uv.set_design_variables(wing.dt, R.Constant(wing.u_inf, wing.rho), z0, hg0)
    st = uv.solve_static()
    return uv, st, OL.LinearUVLMRef(uv, st, wake_type)


def rigid_projections(xp, zeta_ref, ea_x):
    """A rigid heave h and pitch theta (about the y axis through x = ea_x) of the reference
    lattice as the linear model's input projection, and the total lift and the pitching
    moment about that axis as its output projection, written against an array module xp
    (jax.numpy for the reference, numpy for the product's tests).  Returns (arg_names, arg_sizes, to_zeta,
    out_size, to_output)."""
    z = np.asarray(zeta_ref, float)

    def to_zeta(hp_vec, hp_dot_vec):
        h, th = hp_vec[0], hp_vec[1]
        hd, thd = hp_dot_vec[0], hp_dot_vec[1]
        dx, dz = z[..., 0] - ea_x, z[..., 2]
        c, s_ = xp.cos(th), xp.sin(th)
        x = ea_x + c * dx + s_ * dz
        zz = -s_ * dx + c * dz + h
        zeta = xp.stack([x, xp.asarray(z[..., 1]), zz], axis=-1)
        xd = thd * (-s_ * dx + c * dz)
        zd = hd + thd * (-c * dx - s_ * dz)
        zeta_dot = xp.stack([xd, xp.zeros_like(xd), zd], axis=-1)
        return zeta.ravel(), zeta_dot.ravel()

    def to_output(fs, fu):
        f = fs if fu is None else fs + fu
        f = f.reshape(-1, 3)
        arm = z.reshape(-1, 3)[:, 0] - ea_x
        return xp.stack([xp.sum(f[:, 2]), -xp.sum(arm * f[:, 2])])

    return ("hp_vec", "hp_dot_vec"), (2, 2), to_zeta, 2, to_output


def projections(g):
    """The product's LinearInputProjection / LinearOutputProjection of a projected golden
    case (the same rigid heave-pitch and lift-moment maps, in numpy)."""
    from flapjax_b200.linear import LinearInputProjection, LinearOutputProjection

    names, sizes, to_zeta, out_size, to_output = rigid_projections(np, g["ref_zeta_b"], float(g["ea_x"]))
    ip = LinearInputProjection(arg_names=names, arg_sizes=sizes, arg_refs=(np.zeros(2), np.zeros(2)),
                               to_zeta=to_zeta)
    op = LinearOutputProjection(name="lift_moment", size=out_size, to_output=to_output)
    return ip, op
