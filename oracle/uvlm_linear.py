"""CPU restatement of the reference's linearised UVLM (aero/linear/linear_uvlm.py) and its
discrete state-space system (utils/linear.py:673-822), for checking the CUDA-assembled
linear model.  Test infrastructure: only tests import this module.

The linear model steps the nonlinear UVLM once from states x_n to x_{n+1} with the inputs
of step n+1 (``LinearUVLM.step`` :324-429) and takes its Jacobians at a reference
(steady) solution; the reference computes them with jax.jacrev, here they are central
differences of the restated step.  Only the (residual, argument) pairs that the
reference differentiates (``compute_jacobians`` :499-621) are filled; the other blocks
stay zero, as ``construct_named_block_jacobian`` (algebra/array_utils.py:406-445) leaves
them.

Vectors follow the reference's slice order (``_make_*_slices`` :248-322), each block the
concatenation of its surfaces:

* inputs  u = [zeta_b, zeta_b_dot, nu_b, nu_w]
* states  x = [gamma_b, gamma_w, gamma_b_nm1, zeta_w, zeta_b]  (the last two only for the
  prescribed and free wake types, gamma_b_nm1 only with the unsteady force)
* outputs y = [f_steady, f_unsteady]
"""
from __future__ import annotations

import numpy as np

from oracle import uvlm_ref as R

# compute_jacobians (:499-621): residual -> the arguments it differentiates
_STATE_ARG = {"gamma_b": "gamma_b", "gamma_w": "gamma_w", "gamma_b_nm1": "gamma_b_nm1", "zeta_w": "zeta_w",
              "zeta_b": "zeta_b"}


def diff_lists(wake_type, bound_upwash=True, wake_upwash=True, unsteady_force=True):
    prescribed = wake_type in ("prescribed", "free")
    g_b = ["x:gamma_b", "x:gamma_w", "u:zeta_b", "u:zeta_b_dot"]
    if prescribed:
        g_b += ["x:zeta_w", "x:zeta_b"]
    if bound_upwash:
        g_b.append("u:nu_b")
    if wake_upwash:
        g_b.append("u:nu_w")
    out = {"gamma_b": g_b, "gamma_w": ["x:gamma_b", "x:gamma_w"]}
    if prescribed:
        z_w = ["x:zeta_w", "u:zeta_b"]
        if wake_upwash:
            z_w.append("u:nu_w")
        if wake_type == "free":
            z_w += ["x:gamma_b", "x:gamma_w"]
        out["zeta_w"] = z_w
    if unsteady_force:
        out["gamma_b_nm1"] = ["x:gamma_b"]
    if prescribed:
        out["zeta_b"] = ["u:zeta_b"]
    f_s = ["x:gamma_b", "x:gamma_w", "u:zeta_b", "u:zeta_b_dot"]
    if prescribed:
        f_s.append("x:zeta_w")
    if bound_upwash:
        f_s.append("u:nu_b")
    out["f_steady"] = f_s
    if unsteady_force:
        out["f_unsteady"] = ["x:gamma_b", "x:gamma_b_nm1", "u:zeta_b"]
    return out


class LinearSystemRef:
    """``LinearSystem`` utils/linear.py:673-822 (discrete time)."""

    def __init__(self, a, b, c, d, dt, removed_u_np1=False):
        self.a, self.b, self.c, self.d = a, b, c, d
        self.dt = dt
        self.removed_u_np1 = removed_u_np1

    def remove_u_np1(self):
        """:714-724: D <- C B + D, B <- A B."""
        if not self.removed_u_np1:
            self.d = self.c @ self.b + self.d
            self.b = self.a @ self.b
            self.removed_u_np1 = True

    def run(self, u, x0=None):
        """:775-822: x_n = A x_{n-1} + B u_n (u_{n-1} once u_np1 is removed), x_0 = x0;
        y_n = C x_n + D u_n."""
        n_t = u.shape[0]
        x = np.zeros((n_t, self.a.shape[0]))
        if x0 is not None:
            x[0] = x0
        for i in range(1, n_t):
            uu = u[i - 1] if self.removed_u_np1 else u[i]
            x[i] = self.a @ x[i - 1] + self.b @ uu
        y = x @ self.c.T + u @ self.d.T
        return x, y


class LinearUVLMRef:
    """``LinearUVLM`` aero/linear/linear_uvlm.py:81-429 over an ``oracle.uvlm_ref.UVLMRef``
    and its static solution (a ``Case`` of one step)."""

    def __init__(self, uv, static_case, wake_type="frozen", bound_upwash=True, wake_upwash=True,
                 unsteady_force=True):
        if wake_type not in ("frozen", "prescribed", "free"):
            raise ValueError(f"wake_type {wake_type!r}")
        self.uv = uv
        self.wake_type = wake_type
        self.prescribed = wake_type in ("prescribed", "free")
        self.bound_upwash, self.wake_upwash, self.unsteady_force = bound_upwash, wake_upwash, unsteady_force
        sc = static_case
        self.ref = {k: [np.asarray(a[0], float) for a in getattr(sc, k)]
                    for k in ("zeta_b", "zeta_w", "gamma_b", "gamma_w", "f_steady")}
        self.ref["zeta_b_dot"] = [np.zeros_like(z) for z in self.ref["zeta_b"]]
        self.ref["gamma_b_dot"] = [np.zeros_like(g) for g in self.ref["gamma_b"]]
        self.t = float(sc.t[0])
        # the linear model's own force kernel is the cutoff kernel (:155-160), whose radius
        # is the module constant R_CUTOFF (aero/utils.py:648)
        self.force_r_cut = uv.r_cut if uv.kernel == R.KERNEL_CUTOFF else R.R_CUTOFF
        zb, zw, gb = self.ref["zeta_b"], self.ref["zeta_w"], self.ref["gamma_b"]
        self.u_blocks = [("zeta_b", zb), ("zeta_b_dot", zb)]
        if bound_upwash:
            self.u_blocks.append(("nu_b", zb))
        if wake_upwash:
            self.u_blocks.append(("nu_w", zw))
        self.x_blocks = [("gamma_b", gb), ("gamma_w", self.ref["gamma_w"])]
        if unsteady_force:
            self.x_blocks.append(("gamma_b_nm1", gb))
        if self.prescribed:
            self.x_blocks += [("zeta_w", zw), ("zeta_b", zb)]
        self.y_blocks = [("f_steady", zb)]
        if unsteady_force:
            self.y_blocks.append(("f_unsteady", zb))

    # -- vectors ------------------------------------------------------------------------
    @staticmethod
    def _size(blocks):
        return sum(sum(a.size for a in t) for _, t in blocks)

    @property
    def n_inputs(self):
        return self._size(self.u_blocks)

    @property
    def n_states(self):
        return self._size(self.x_blocks)

    @property
    def n_outputs(self):
        return self._size(self.y_blocks)

    @staticmethod
    def pack(blocks, d):
        return np.concatenate([np.concatenate([np.ravel(a) for a in d[k]]) for k, _ in blocks])

    @staticmethod
    def unpack(blocks, v):
        out, off = {}, 0
        for k, tmpl in blocks:
            out[k] = []
            for a in tmpl:
                out[k].append(np.asarray(v[off:off + a.size]).reshape(a.shape))
                off += a.size
        return out

    def reference_vectors(self):
        u = {"zeta_b": self.ref["zeta_b"], "zeta_b_dot": self.ref["zeta_b_dot"],
             "nu_b": [np.zeros_like(z) for z in self.ref["zeta_b"]],
             "nu_w": [np.zeros_like(z) for z in self.ref["zeta_w"]]}
        x = {"gamma_b": self.ref["gamma_b"], "gamma_w": self.ref["gamma_w"], "gamma_b_nm1": self.ref["gamma_b"],
             "zeta_w": self.ref["zeta_w"], "zeta_b": self.ref["zeta_b"]}
        return self.pack(self.u_blocks, u), self.pack(self.x_blocks, x)

    # -- the nonlinear step (:324-429) ---------------------------------------------------
    def step(self, u_vec, x_vec, arc_held=None, arc_record=None):
        """One nonlinear step; with a variable wake, ``arc_held`` (one array per surface
        with delta_w, in surface order) stands for the arc lengths that the reference's
        stop_gradient holds, and ``arc_record`` receives the arc lengths used."""
        uv, ref = self.uv, self.ref
        u = self.unpack(self.u_blocks, u_vec)
        x = self.unpack(self.x_blocks, x_vec)
        zb1, zbd1 = u["zeta_b"], u["zeta_b_dot"]
        nu_b = u.get("nu_b")
        nu_w = u.get("nu_w")
        gb_n, gw_n = x["gamma_b"], x["gamma_w"]
        if self.unsteady_force:
            gbd_n = [(a - b) / uv.dt for a, b in zip(gb_n, x["gamma_b_nm1"])]
        else:
            gbd_n = ref["gamma_b_dot"]
        if self.prescribed:
            zb_n, zw_n = x["zeta_b"], x["zeta_w"]
        else:
            zb_n, zw_n = ref["zeta_b"], ref["zeta_w"]
        q_n = (gb_n, gw_n, ref["gamma_b_dot"], zw_n)
        held = None
        if arc_held is not None:
            it = iter(arc_held)
            held = [None if d is None else next(it) for d in uv.delta_w]
        out = uv.base_solve_from_grid(q_n, self.t, zb1, zb_n, zbd1, False, nu_b=nu_b, nu_w=nu_w, arc_held=held,
                                      arc_record=arc_record)
        ff = uv.flowfield

        def v_out(x_):
            return ff(x_, self.t) + R.compute_v_ind(x_, [*zb1, *zw_n], [*gb_n, *gw_n], R.KERNEL_CUTOFF, uv.mirror,
                                                    self.force_r_cut)

        f_s = R.calculate_steady_forcing(zb1, zbd1, gb_n, gw_n, ff.rho, v_out, nu_b if self.bound_upwash else None)
        x1 = {"gamma_b": out["gamma_b"], "gamma_w": out["gamma_w"], "gamma_b_nm1": gb_n, "zeta_w": out["zeta_w"],
              "zeta_b": zb1}
        y0 = {"f_steady": f_s}
        if self.unsteady_force:
            y0["f_unsteady"] = [R.split_to_vertex(ff.rho * g[..., None] * R.compute_surf_nc(z), (0, 1))
                                for g, z in zip(gbd_n, zb1)]
        return self.pack(self.x_blocks, x1), self.pack(self.y_blocks, y0)

    # -- Jacobians by central differences -----------------------------------------------
    def _offsets(self, blocks):
        off, o = {}, 0
        for k, t in blocks:
            n = sum(a.size for a in t)
            off[k] = (o, o + n)
            o += n
        return off

    def linearise(self, h=1e-6):
        """(A, B, C, D) with the reference's differentiated blocks only."""
        u0, x0 = self.reference_vectors()
        arcs = []
        self.step(u0, x0, arc_record=arcs)  # the variable wake's arc lengths at the reference point
        held = arcs if arcs else None
        xo, uo, yo = self._offsets(self.x_blocks), self._offsets(self.u_blocks), self._offsets(self.y_blocks)
        lists = diff_lists(self.wake_type, self.bound_upwash, self.wake_upwash, self.unsteady_force)
        args = sorted({a for v in lists.values() for a in v})
        col = {}
        for a in args:
            kind, name = a.split(":")
            lo, hi = (xo if kind == "x" else uo)[name]
            jx = np.zeros((x0.size, hi - lo))
            jy = np.zeros((self.n_outputs, hi - lo))
            for j in range(hi - lo):
                up, xp, um, xm = u0.copy(), x0.copy(), u0.copy(), x0.copy()
                if kind == "x":
                    xp[lo + j] += h
                    xm[lo + j] -= h
                else:
                    up[lo + j] += h
                    um[lo + j] -= h
                sxp, syp = self.step(up, xp, held)
                sxm, sym = self.step(um, xm, held)
                jx[:, j] = (sxp - sxm) / (2 * h)
                jy[:, j] = (syp - sym) / (2 * h)
            col[a] = (jx, jy)
        A = np.zeros((self.n_states, self.n_states))
        B = np.zeros((self.n_states, self.n_inputs))
        C = np.zeros((self.n_outputs, self.n_states))
        D = np.zeros((self.n_outputs, self.n_inputs))
        for res, diff in lists.items():
            is_out = res in ("f_steady", "f_unsteady")
            r0, r1 = (yo if is_out else xo)[res]
            for a in diff:
                kind, name = a.split(":")
                c0, c1 = (xo if kind == "x" else uo)[name]
                blk = col[a][1 if is_out else 0][r0:r1]
                tgt = (C if kind == "x" else D) if is_out else (A if kind == "x" else B)
                tgt[r0:r1, c0:c1] = blk
        return LinearSystemRef(A, B, C, D, self.uv.dt)
