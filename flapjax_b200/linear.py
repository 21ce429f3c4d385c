"""The linearised UVLM (aero/linear/linear_uvlm.py) and its discrete state-space system
(utils/linear.py:673-822), assembled on the device.

The reference linearises one UVLM step (``LinearUVLM.step``, :324-429: the nonlinear
step from states x_n to x_{n+1} with the inputs of step n+1) about a steady reference
solution by ``jax.jacrev`` of each residual with respect to the arguments listed in
``compute_jacobians`` (:499-621), and assembles A, B, C, D from the blocks
(``linearise``, :727-829).  Here the same blocks come from the chain rule written out,
with every pairwise Biot-Savart term on the GPU:

* the bound circulation of step n+1 is Gamma_b = A(zeta_b)^-1 Phi, Phi = -n . V(c) with
  V the total velocity at the collocation points (free stream, -c_dot, induced velocity
  of the new wake and the bound upwash input).  Holding Gamma_b at its value the
  derivative of A Gamma_b folds into the bound lattice's share of V, so
  dGamma_b = A^-1 dPhi, and dPhi needs
    - the ring influence of the wake at c (fj_ring_influence, normals): the wake
      circulation shifted from the states;
    - the vertex Jacobians of the wake and bound lattices at c (fj_vertex_jacobian,
      normals): the trailing-edge row of the new wake is the input lattice's, the
      wake upwash moves every wake vertex, the bound lattice moves its own sources;
    - n^T grad V at c (fj_vind_vjp with cotangent n) and the normals' derivative;
    - for a free wake, the convection velocity's ring and vertex Jacobians and its
      gradient at the convected vertices;
  and A^-1 is applied to all columns at once (fj_lu_factor, fj_lu_solve_many);
* the wake rows shift and convect, and a variable wake is re-discretised with fixed
  interpolation weights (aero/utils.py:400-500, ``_WakeMap``);
* the steady force f = rho g (v_rel x r) per filament (aero/utils.py:126-223, the linear
  model's own cutoff kernel :155-160) is differentiated through its strength g, the
  relative velocity at the midpoint (ring and vertex Jacobians of the bound and wake
  lattices at the midpoints, 3 rows each; the velocity gradient there) and the filament
  vector, then split to the vertices; the unsteady force through Gamma_dot.

Blocks the reference does not differentiate stay zero.  Vectors follow the reference's
slice order, each block the concatenation of its surfaces:

* inputs  u = [zeta_b, zeta_b_dot, nu_b, nu_w]
* states  x = [gamma_b, gamma_w, gamma_b_nm1, zeta_w, zeta_b]  (zeta_w, zeta_b only for
  the prescribed and free wake types; gamma_b_nm1 only with the unsteady force)
* outputs y = [f_steady, f_unsteady]

Scope: FP64, epsilon or cutoff kernel for the UVLM's own sums, any number of surfaces,
mirror images, Constant or 1-cos gust flow, uniform or variable wake (``delta_w``: the
re-discretisation with its arc lengths held at the reference point, as the reference's
``linearise_variable_wake`` holds them).  The
reference point is a steady solution (the static solve), so Gamma_dot there is zero and
the unsteady force has no geometric derivative.
"""
from __future__ import annotations

import ctypes as C
import warnings
from collections.abc import Callable
from dataclasses import dataclass

import numpy as np

from . import _lib
from .adjoint import _flow_T
from .kernels import R_CUTOFF
from .runtime import device_of

WAKE_TYPES = ("frozen", "prescribed", "free")


@dataclass
class LinearInputProjection:
    """Lattice coordinates and velocities from a lower-dimensional input space, e.g. beam
    coordinates (aero/linear/linear_uvlm.py:48-63).  ``to_zeta(**{name: vec})`` returns
    the total ``(zeta_b_vec, zeta_b_dot_vec)`` (surfaces concatenated, raveled).  The
    reference differentiates ``to_zeta`` with jax; here ``jacobian(**{name: vec})`` gives
    ``(d zeta_b / d q, d zeta_b_dot / d q)`` over the concatenated arguments q when it is
    supplied, else central differences of ``to_zeta`` (step ``fd_step``) at ``arg_refs``."""

    arg_names: tuple
    arg_sizes: tuple
    arg_refs: tuple
    to_zeta: Callable
    jacobian: Callable | None = None
    fd_step: float = 1e-6


@dataclass
class LinearOutputProjection:
    """Forces onto one output space (aero/linear/linear_uvlm.py:65-78):
    ``to_output(f_steady_vec, f_unsteady_vec | None) -> vector of length size``.  Its
    Jacobian is ``jacobian(f_steady_vec, f_unsteady_vec)`` -> ``(d out / d f_steady,
    d out / d f_unsteady or None)`` when supplied, else central differences (step
    ``fd_step``) at the reference forces."""

    name: str
    size: int
    to_output: Callable
    jacobian: Callable | None = None
    fd_step: float = 1e-6


@dataclass
class AeroInputUnflattened:
    """Inputs per surface, time-batched in ``run`` (aero/linear/data_structures.py:16-22):
    zeta_b and zeta_b_dot (n_tstep, m+1, n+1, 3), nu_b the same or None, nu_w
    (n_tstep, m_star+1, n+1, 3) or None."""

    zeta_b: list
    zeta_b_dot: list
    nu_b: list | None = None
    nu_w: list | None = None


@dataclass
class AeroStateUnflattened:
    """States per surface (aero/linear/data_structures.py:24-31)."""

    gamma_b: list
    gamma_w: list
    gamma_b_nm1: list | None = None
    zeta_w: list | None = None
    zeta_b: list | None = None


@dataclass
class AeroOutputUnflattened:
    """Outputs per surface (aero/linear/data_structures.py:33-36)."""

    f_steady: list
    f_unsteady: list | None = None


@dataclass
class AeroLinearResult:
    """A linear run (aero/linear/data_structures.py:39-): perturbations u_t, x_t, y_t and
    totals (reference + perturbation), per surface with a leading time axis."""

    reference: object
    u_t: AeroInputUnflattened
    x_t: AeroStateUnflattened
    y_t: AeroOutputUnflattened
    u_t_tot: AeroInputUnflattened
    x_t_tot: AeroStateUnflattened
    y_t_tot: AeroOutputUnflattened
    n_tstep: int
    n_surf: int
    t: np.ndarray


def _fd_columns(fun, x0, h):
    """Central-difference Jacobian of fun (vector -> tuple of vectors) at x0: one matrix
    per output."""
    x0 = np.asarray(x0, np.float64)
    cols = None
    for j in range(x0.size):
        xp, xm = x0.copy(), x0.copy()
        xp[j] += h
        xm[j] -= h
        fp, fm = fun(xp), fun(xm)
        if cols is None:
            cols = [np.zeros((np.size(a), x0.size)) for a in fp]
        for c, a, b in zip(cols, fp, fm):
            c[:, j] = (np.ravel(a) - np.ravel(b)) / (2 * h)
    return cols


# ---------------------------------------------------------------------------------------
# the state-space system
# ---------------------------------------------------------------------------------------
class LinearSystem:
    """x_n = A x_{n-1} + B u_n, y_n = C x_n + D u_n (utils/linear.py:673-822), device
    tensors (FP64)."""

    def __init__(self, a, b, c, d, dt, removed_u_np1: bool = False):
        self.a, self.b, self.c, self.d = a, b, c, d
        self.dt = float(dt)
        self.n_inputs = int(b.shape[1])
        self.n_states = int(a.shape[0])
        self.n_outputs = int(c.shape[0])
        self.continuous_time = False
        self.removed_u_np1 = bool(removed_u_np1)

    def remove_u_np1(self) -> None:
        """:714-724: D <- C B + D and B <- A B (inputs of step n instead of n+1)."""
        if self.removed_u_np1:
            warnings.warn("u_np1 has already been removed from the system. Skipping.")
            return
        self.d = self.c @ self.b + self.d
        self.b = self.a @ self.b
        self.removed_u_np1 = True

    def run(self, u, x0=None):
        """:775-822: state and output histories for the input history u (n_tstep, n_inputs),
        from x0 (zero if None).  Returns device tensors (n_tstep, n_states), (n_tstep,
        n_outputs)."""
        import torch

        dev = self.a.device
        if dev.type != "cuda":
            raise RuntimeError("LinearSystem.run marches on the GPU (fj_lti_march): its matrices must be CUDA "
                               "tensors")
        u = torch.as_tensor(np.asarray(u) if not torch.is_tensor(u) else u, dtype=torch.float64).to(dev)
        if u.ndim != 2 or u.shape[1] != self.n_inputs:
            raise ValueError(f"Expected shape (None, {self.n_inputs}), but got shape {tuple(u.shape)}.Issue with "
                             f"input 'u'")
        n_t = u.shape[0]
        x = torch.zeros((n_t, self.n_states), dtype=torch.float64, device=dev)
        if x0 is not None:
            x0 = torch.as_tensor(np.asarray(x0) if not torch.is_tensor(x0) else x0, dtype=torch.float64).to(dev)
            if tuple(x0.shape) != (self.n_states,):
                raise ValueError(f"Expected shape ({self.n_states},), but got shape {tuple(x0.shape)}.Issue with "
                                 f"input 'x0'")
            x[0] = x0
        bu = (u @ self.b.T).contiguous()  # every step's input term in one product
        a = self.a.contiguous()
        _lib.call("fj_lti_march", a.data_ptr(), self.n_states, bu.data_ptr(), bu.stride(0), x.data_ptr(), n_t,
                  1 if self.removed_u_np1 else 0, torch.cuda.current_stream(dev).cuda_stream)
        y = x @ self.c.T + u @ self.d.T
        return x, y


# ---------------------------------------------------------------------------------------
# device operations (the C ABI)
# ---------------------------------------------------------------------------------------
class _CudaOps:
    """The pairwise sums, Jacobians and solves of the assembly, on the GPU (FP64)."""

    def __init__(self, device, mirror):
        import torch

        self.torch = torch
        self.dev = device_of(device)
        self._mir = None if mirror is None else tuple(
            (C.c_double * 3)(*np.asarray(v, dtype=np.float64).tolist()) for v in mirror)
        self._ws = {}

    def tensor(self, a):
        return self.torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(self.dev)

    def zeros(self, *shape):
        return self.torch.zeros(shape, dtype=self.torch.float64, device=self.dev)

    def _wsb(self, key, nbytes):
        w = self._ws.get(key)
        if w is None or w.numel() < nbytes:
            w = self.torch.empty(max(int(nbytes), 1), dtype=self.torch.uint8, device=self.dev)
            self._ws[key] = w
        return w

    def _stream(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def _mirror(self):
        return self._mir if self._mir is not None else (None, None)

    def ring(self, out, col0, targets, normals, zeta, kernel, r_cut):
        """out[:, col0 + r] <- d v(targets) / d gamma_r of lattice zeta (rows: 1 per target
        with normals, else 3)."""
        mp, mn = self._mirror()
        _lib.call("fj_ring_influence", targets.data_ptr(), targets.shape[0],
                  None if normals is None else normals.data_ptr(), zeta.data_ptr(), zeta.shape[0] - 1,
                  zeta.shape[1] - 1, mp, mn, kernel, r_cut, out.data_ptr() + 8 * col0, out.stride(0),
                  self._stream())

    def vertex(self, out, col0, targets, normals, zeta, gamma, kernel, r_cut):
        """out[:, col0 + 3v + b] <- d v(targets) / d zeta_vb for circulations gamma."""
        mp, mn = self._mirror()
        _lib.call("fj_vertex_jacobian", targets.data_ptr(), targets.shape[0],
                  None if normals is None else normals.data_ptr(), zeta.data_ptr(), gamma.data_ptr(),
                  zeta.shape[0] - 1, zeta.shape[1] - 1, mp, mn, kernel, r_cut, out.data_ptr() + 8 * col0,
                  out.stride(0), self._stream())

    def _lats(self, lats):
        n = len(lats)
        return ((C.c_void_p * n)(*[z.data_ptr() for z, _ in lats]), (C.c_void_p * n)(*[g.data_ptr() for _, g in lats]),
                (C.c_int * n)(*[z.shape[0] - 1 for z, _ in lats]), (C.c_int * n)(*[z.shape[1] - 1 for z, _ in lats]))

    def vind(self, targets, lats, kernel, r_cut):
        zp, gp, rows, cols = self._lats(lats)
        mp, mn = self._mirror()
        nb = C.c_size_t()
        _lib.call("fj_vind_workspace_size", targets.shape[0], rows, cols, len(lats), int(self._mir is not None),
                  _lib.FJ_PREC_FP64, C.byref(nb))
        ws = self._wsb("vind", nb.value)
        out = self.torch.empty_like(targets)
        _lib.call("fj_vind", targets.data_ptr(), targets.shape[0], zp, gp, rows, cols, len(lats), mp, mn, kernel,
                  r_cut, _lib.FJ_PREC_FP64, out.data_ptr(), ws.data_ptr(), ws.numel(), self._stream())
        return out

    def vind_grad_t(self, targets, lats, kernel, r_cut, lam):
        """sum_s d(lam_t . v(x_t))/dx_t per target (the target share of fj_vind_vjp)."""
        zp, gp, rows, cols = self._lats(lats)
        mp, mn = self._mirror()
        nb = C.c_size_t()
        _lib.call("fj_vind_vjp_workspace_size", targets.shape[0], rows, cols, len(lats), int(self._mir is not None),
                  C.byref(nb))
        ws = self._wsb("vjp", nb.value)
        out = self.torch.zeros_like(targets)
        _lib.call("fj_vind_vjp", targets.data_ptr(), targets.shape[0], zp, gp, rows, cols, len(lats), mp, mn,
                  kernel, r_cut, lam.data_ptr(), out.data_ptr(), None, None, ws.data_ptr(), ws.numel(),
                  self._stream())
        return out

    def aic_factor(self, zetas_b, kernel, r_cut):
        k = len(zetas_b)
        zp = (C.c_void_p * k)(*[z.data_ptr() for z in zetas_b])
        ms = (C.c_int * k)(*[z.shape[0] - 1 for z in zetas_b])
        ns = (C.c_int * k)(*[z.shape[1] - 1 for z in zetas_b])
        nb = sum((z.shape[0] - 1) * (z.shape[1] - 1) for z in zetas_b)
        a = self.torch.empty((nb, nb), dtype=self.torch.float64, device=self.dev)
        w = C.c_size_t()
        _lib.call("fj_aic_workspace_size", ms, ns, k, C.byref(w))
        ws = self._wsb("aic", w.value)
        mp, mn = self._mirror()
        s = self._stream()
        _lib.call("fj_aic_assemble", zp, ms, ns, k, None, (C.c_int * k)(*([0] * k)), mp, mn, kernel, r_cut,
                  a.data_ptr(), ws.data_ptr(), ws.numel(), s)
        piv = self.torch.empty(nb, dtype=self.torch.int32, device=self.dev)
        _lib.call("fj_lu_workspace_size", nb, C.byref(w))
        wl = self._wsb("lu", w.value)
        _lib.call("fj_lu_factor", a.data_ptr(), nb, piv.data_ptr(), wl.data_ptr(), wl.numel(), s)
        return a, piv

    def solve(self, lu, piv, b):
        n = piv.numel()
        w = C.c_size_t()
        _lib.call("fj_lu_workspace_size", n, C.byref(w))
        wl = self._wsb("lu", w.value)
        x = b.clone().contiguous()
        _lib.call("fj_lu_solve", lu.data_ptr(), n, piv.data_ptr(), x.data_ptr(), wl.data_ptr(), wl.numel(),
                  self._stream())
        return x

    def solve_many(self, lu, piv, b):
        """b <- A^-1 b in place for the columns of the row-major (n, m) b."""
        n = piv.numel()
        w = C.c_size_t()
        _lib.call("fj_lu_solve_many_workspace_size", n, b.shape[1], C.byref(w))
        ws = self._wsb("many", w.value)
        _lib.call("fj_lu_solve_many", lu.data_ptr(), n, piv.data_ptr(), b.data_ptr(), b.shape[1], b.stride(0),
                  ws.data_ptr(), ws.numel(), self._stream())


# ---------------------------------------------------------------------------------------
# geometry bookkeeping (host)
# ---------------------------------------------------------------------------------------
def _skew(v):
    """[v]x per row: (..., 3) -> (..., 3, 3) with [v]x w = v x w."""
    o = np.zeros(v.shape[:-1] + (3, 3))
    o[..., 0, 1], o[..., 0, 2] = -v[..., 2], v[..., 1]
    o[..., 1, 0], o[..., 1, 2] = v[..., 2], -v[..., 0]
    o[..., 2, 0], o[..., 2, 1] = -v[..., 1], v[..., 0]
    return o


def _flow_grad(ff, x, t):
    """d u_a / d x_b of the flow field at points x (..., 3) -> (..., 3, 3)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros(x.shape + (3,))
    for a in range(3):
        e = np.zeros(3)
        e[a] = 1.0
        out[..., a, :] = _flow_T(ff, x, t, np.broadcast_to(e, x.shape))
    return out


class _Layout:
    """Offsets of every block of the state, input and output vectors."""

    def __init__(self, dims, wake_type, bound_upwash, wake_upwash, unsteady_force):
        self.dims = dims  # per surface (m, n, m_star)
        self.nb = [m * n for m, n, _ in dims]
        self.nw = [w * n for _, n, w in dims]
        self.nvb = [(m + 1) * (n + 1) for m, n, _ in dims]
        self.nvw = [(w + 1) * (n + 1) for _, n, w in dims]
        cum = lambda v: np.concatenate([[0], np.cumsum(v)]).astype(np.int64)
        self.o_gb, self.o_gw, self.o_vb, self.o_vw = cum(self.nb), cum(self.nw), cum(self.nvb), cum(self.nvw)
        NB, NW, NVB, NVW = int(self.o_gb[-1]), int(self.o_gw[-1]), int(self.o_vb[-1]), int(self.o_vw[-1])
        self.NB, self.NW, self.NVB, self.NVW = NB, NW, NVB, NVW
        prescribed = wake_type in ("prescribed", "free")
        x = [("gamma_b", NB), ("gamma_w", NW)]
        if unsteady_force:
            x.append(("gamma_b_nm1", NB))
        if prescribed:
            x += [("zeta_w", 3 * NVW), ("zeta_b", 3 * NVB)]
        u = [("zeta_b", 3 * NVB), ("zeta_b_dot", 3 * NVB)]
        if bound_upwash:
            u.append(("nu_b", 3 * NVB))
        if wake_upwash:
            u.append(("nu_w", 3 * NVW))
        y = [("f_steady", 3 * NVB)]
        if unsteady_force:
            y.append(("f_unsteady", 3 * NVB))

        def offs(blocks):
            o, d = 0, {}
            for k, n in blocks:
                d[k] = (o, o + n)
                o += n
            return d, o

        self.x, self.n_states = offs(x)
        self.u, self.n_inputs = offs(u)
        self.y, self.n_outputs = offs(y)
        self.x_blocks, self.u_blocks, self.y_blocks = x, u, y

    # columns of [states | inputs]
    def col(self, kind, name):
        if kind == "x":
            return self.x.get(name)
        r = self.u.get(name)
        return None if r is None else (self.n_states + r[0], self.n_states + r[1])


def _diff_lists(wake_type, bound_upwash, wake_upwash, unsteady_force):
    """compute_jacobians (:499-621): residual -> differentiated arguments."""
    prescribed = wake_type in ("prescribed", "free")
    g_b = ["x:gamma_b", "x:gamma_w", "u:zeta_b", "u:zeta_b_dot"] + (["x:zeta_w", "x:zeta_b"] if prescribed else [])
    g_b += (["u:nu_b"] if bound_upwash else []) + (["u:nu_w"] if wake_upwash else [])
    out = {"gamma_b": g_b, "gamma_w": ["x:gamma_b", "x:gamma_w"]}
    if prescribed:
        out["zeta_w"] = ["x:zeta_w", "u:zeta_b"] + (["u:nu_w"] if wake_upwash else []) + (
            ["x:gamma_b", "x:gamma_w"] if wake_type == "free" else [])
    if unsteady_force:
        out["gamma_b_nm1"] = ["x:gamma_b"]
    if prescribed:
        out["zeta_b"] = ["u:zeta_b"]
    out["f_steady"] = ["x:gamma_b", "x:gamma_w", "u:zeta_b", "u:zeta_b_dot"] + (
        ["x:zeta_w"] if prescribed else []) + (["u:nu_b"] if bound_upwash else [])
    if unsteady_force:
        out["f_unsteady"] = ["x:gamma_b", "x:gamma_b_nm1", "u:zeta_b"]
    return out


# ---------------------------------------------------------------------------------------
# assembly
# ---------------------------------------------------------------------------------------
def _interp_weights(xq, xp):
    """W with W @ fp = interp(xq, xp, fp) for increasing xp (jnp.interp, as
    aero/utils.py:480-491 calls it): end values held outside [xp[0], xp[-1]], linear
    between the bracketing nodes inside."""
    w = np.zeros((len(xq), len(xp)))
    last = len(xp) - 1
    for q, x in enumerate(xq):
        if not x >= xp[0]:
            w[q, 0] = 1.0
        elif x >= xp[last]:
            w[q, last] = 1.0
        else:
            j = int(np.searchsorted(xp, x, side="right")) - 1
            t = (x - xp[j]) / (xp[j + 1] - xp[j])
            w[q, j] += 1.0 - t
            w[q, j + 1] += t
    return w


class _WakeMap:
    """The wake of step n+1 from step n for one surface (aero/utils.py:400-500), per
    spanwise column: zeta_w1 = Wz X and gamma_w1 = Wg G, with X = [trailing edge of step
    n+1; convected vertex rows of step n] and G = [trailing-edge circulation of step n;
    wake circulation rows of step n].  Uniform wake: rows 0..W-1 convect, G holds rows
    0..W-2, and Wz, Wg are identities.  Variable wake (delta_w): every row convects, G
    holds every row, and Wz, Wg re-discretise onto delta_w with the arc lengths of the
    reference point, held as the linear model's stop_gradient holds them
    (``linearise_variable_wake``, :465-468)."""

    def __init__(self, n, w, delta_w, x_ref=None):
        var = delta_w is not None and w > 0
        self.n_conv_rows = w + 1 if var else w
        self.n_x = self.n_conv_rows + 1
        self.n_g = w + 1 if var else w
        if not var:
            self.wz = np.broadcast_to(np.eye(w + 1), (n + 1, w + 1, w + 1))
            self.wg = np.broadcast_to(np.eye(w), (n, w, w))
            return
        if x_ref is None:  # row counts only
            return
        seg = np.linalg.norm(x_ref[1:] - x_ref[:-1], axis=-1)
        arc = np.concatenate([np.zeros((1, n + 1)), np.cumsum(seg, axis=0)], axis=0)       # (W+2, n+1)
        arc_g = 0.5 * (0.5 * (arc[:-1, :-1] + arc[1:, :-1]) + 0.5 * (arc[:-1, 1:] + arc[1:, 1:]))
        s_disc = np.concatenate([np.zeros(1), np.cumsum(np.asarray(delta_w, np.float64))])
        sg_disc = 0.5 * (s_disc[:-1] + s_disc[1:])
        self.wz = np.stack([_interp_weights(s_disc, arc[:, j]) for j in range(n + 1)])       # (n+1, W+1, W+2)
        self.wg = np.stack([_interp_weights(sg_disc, arc_g[:, j]) for j in range(n)])         # (n, W, W+1)

    def apply_z(self, x):
        """(n_x, n+1, ...) -> (W+1, n+1, ...)."""
        return np.einsum("jrs,sj...->rj...", self.wz, x)

    def apply_g(self, g):
        return np.einsum("jrs,sj->rj", self.wg, g)


def _assemble(ops, lay, ref, cfg):
    """Jacobian rows of every residual over the columns [states | inputs].

    ref: host arrays per surface (zeta_b, zeta_w, gamma_b, gamma_w); cfg: wake_type,
    free_wake, kernel, r_cut, force_r_cut, dt, rho, flowfield, t, bound_upwash,
    wake_upwash, unsteady_force, delta_w (per surface or None).  Returns (R_state, R_out), the Jacobians of the next
    states and of the outputs, each (rows, n_states + n_inputs), on the ops' device."""
    torch = ops.torch
    S = len(lay.dims)
    ff, t, dt, rho = cfg["flowfield"], cfg["t"], cfg["dt"], cfg["rho"]
    K, RC, FK, FRC = cfg["kernel"], cfg["r_cut"], _lib.FJ_KERNEL_CUTOFF, cfg["force_r_cut"]
    free = cfg["free_wake"]
    wt = cfg["wake_type"]
    prescribed = wt in ("prescribed", "free")
    ncol = lay.n_states + lay.n_inputs
    lists = _diff_lists(wt, cfg["bound_upwash"], cfg["wake_upwash"], cfg["unsteady_force"])
    Zb = [np.asarray(z, np.float64) for z in ref["zeta_b"]]
    Zw = [np.asarray(z, np.float64) for z in ref["zeta_w"]]
    gb = [np.asarray(g, np.float64) for g in ref["gamma_b"]]
    gw = [np.asarray(g, np.float64) for g in ref["gamma_w"]]
    tZb, tZw = [ops.tensor(z) for z in Zb], [ops.tensor(z) for z in Zw]
    tgb, tgw = [ops.tensor(g) for g in gb], [ops.tensor(g) for g in gw]

    def cols(kind, name):
        return lay.col(kind, name)

    # ---- forward at the reference point -------------------------------------------------
    dws = cfg.get("delta_w") or [None] * S
    maps0 = [_WakeMap(n, w, dw if w > 0 else None) for (m, n, w), dw in zip(lay.dims, dws)]
    conv_pts = [z[:mp.n_conv_rows] for z, mp in zip(Zw, maps0)]          # wake vertex rows that convect
    n_conv = [p.shape[0] * p.shape[1] for p in conv_pts]
    o_conv = np.concatenate([[0], np.cumsum(n_conv)]).astype(np.int64)
    NC = int(o_conv[-1])
    conv_flat = np.concatenate([p.reshape(-1, 3) for p in conv_pts]) if NC else np.zeros((0, 3))
    t_conv = ops.tensor(conv_flat)
    vc = ff(conv_flat, t)
    if free and NC:
        vc = vc + ops.vind(t_conv, list(zip(tZb, tgb)) + list(zip(tZw, tgw)), K, RC).cpu().numpy()
    zw1, gw1, maps = [], [], []
    for s, (m, n, w) in enumerate(lay.dims):
        conv = conv_pts[s] + dt * vc[o_conv[s]:o_conv[s + 1]].reshape(conv_pts[s].shape)
        x_ref = np.concatenate([Zb[s][-1][None], conv], axis=0)
        g_ref = np.concatenate([gb[s][-1][None], gw[s]], axis=0)[:maps0[s].n_g]
        mp = _WakeMap(n, w, dws[s] if w > 0 else None, x_ref)
        maps.append(mp)
        zw1.append(mp.apply_z(x_ref))
        gw1.append(mp.apply_g(g_ref) if w > 0 else gw[s].copy())
    tzw1, tgw1 = [ops.tensor(z) for z in zw1], [ops.tensor(g) for g in gw1]
    c = [0.25 * (z[:-1, :-1] + z[1:, :-1] + z[:-1, 1:] + z[1:, 1:]) for z in Zb]
    d1 = [z[1:, 1:] - z[:-1, :-1] for z in Zb]
    d2 = [z[1:, :-1] - z[:-1, 1:] for z in Zb]
    nc = [np.cross(a, b) for a, b in zip(d1, d2)]
    c_flat = np.concatenate([x.reshape(-1, 3) for x in c])
    n_flat = np.concatenate([x.reshape(-1, 3) for x in nc])
    tc, tn = ops.tensor(c_flat), ops.tensor(n_flat)
    lu, piv = ops.aic_factor(tZb, K, RC)
    wake_lats = [(z, g) for z, g in zip(tzw1, tgw1) if z.shape[0] > 1]
    v_w = ops.vind(tc, wake_lats, K, RC) if wake_lats else torch.zeros_like(tc)
    u_c = ff(c_flat, t)
    rhs = -np.einsum("ij,ij->i", u_c + v_w.cpu().numpy(), n_flat)
    gb1 = ops.solve(lu, piv, ops.tensor(rhs)).cpu().numpy()
    gb1_s = [gb1[lay.o_gb[s]:lay.o_gb[s + 1]].reshape(m, n) for s, (m, n, _) in enumerate(lay.dims)]
    tgb1 = [ops.tensor(g) for g in gb1_s]
    all_lats = list(zip(tZb, tgb1)) + wake_lats
    v_tot = u_c + ops.vind(tc, all_lats, K, RC).cpu().numpy()            # V(c) at the reference point
    g_c = ops.vind_grad_t(tc, all_lats, K, RC, tn).cpu().numpy()         # n^T grad_x V(c)
    g_c += np.einsum("ia,iab->ib", n_flat, _flow_grad(ff, c_flat, t))

    # ---- gamma_b rows: dPhi over all columns, then A^-1 ----------------------------------
    NB = lay.NB
    phi = ops.zeros(NB, ncol)
    rows, cl, vals = [], [], []                                          # local (sparse) terms

    def add(r, cc, v):
        rows.append(np.asarray(r, np.int64).ravel())
        cl.append(np.asarray(cc, np.int64).ravel())
        vals.append(np.asarray(v, np.float64).ravel())

    pw = None
    if wake_lats and any(k in lists["gamma_b"] for k in ("u:zeta_b", "u:nu_w", "x:zeta_w", "x:zeta_b",
                                                         "x:gamma_b", "x:gamma_w")):
        pw = ops.zeros(NB, 3 * lay.NVW)                                   # n . dV(c)/d zeta_w1
        for s in range(S):
            if Zw[s].shape[0] > 1:
                ops.vertex(pw, 3 * int(lay.o_vw[s]), tc, tn, tzw1[s], tgw1[s], K, RC)
    for s, (m, n, w) in enumerate(lay.dims):
        k_, l_ = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
        i_row = lay.o_gb[s] + k_ * n + l_                                 # (m, n) panel rows
        vb = lay.o_vb[s]
        corner = {"00": vb + k_ * (n + 1) + l_, "01": vb + k_ * (n + 1) + l_ + 1,
                  "10": vb + (k_ + 1) * (n + 1) + l_, "11": vb + (k_ + 1) * (n + 1) + l_ + 1}
        ii = i_row.ravel()
        w_i = v_tot[ii]                                                   # V at c_i
        gi = g_c[ii]
        D1, D2 = d1[s].reshape(-1, 3), d2[s].reshape(-1, 3)
        dn = {"11": np.cross(D2, w_i), "00": -np.cross(D2, w_i), "10": np.cross(w_i, D1), "01": -np.cross(w_i, D1)}
        nrm = n_flat[ii]
        zb_c, zbd_c = cols("u", "zeta_b"), cols("u", "zeta_b_dot")
        nub_c = cols("u", "nu_b")
        for key, vv in corner.items():
            vv = vv.ravel()
            for b in range(3):
                # Phi = -n . V(c): normal and collocation point move with the corner
                add(ii, zb_c[0] + 3 * vv + b, -dn[key][:, b] - 0.25 * gi[:, b])
                add(ii, zbd_c[0] + 3 * vv + b, 0.25 * nrm[:, b])          # -n . (-c_dot)
                if nub_c is not None:
                    add(ii, nub_c[0] + 3 * vv + b, -0.25 * nrm[:, b])     # -n . avg4(nu_b)
        # the bound lattice's own sources (circulation held at Gamma_b of step n+1)
        ops.vertex(phi, zb_c[0] + 3 * int(vb), tc, tn, tZb[s], tgb1[s], K, RC)
    phi[:, zb_c[0]:zb_c[1]] *= -1.0
    pw_conv = None
    if pw is not None:
        zb_c = cols("u", "zeta_b")
        gbc, gwc = cols("x", "gamma_b"), cols("x", "gamma_w")
        qw = ops.zeros(NB, lay.NW)                                        # n . dV(c)/d gamma_w1
        for s in range(S):
            if Zw[s].shape[0] > 1:
                ops.ring(qw, int(lay.o_gw[s]), tc, tn, tzw1[s], K, RC)
        conv_parts = []
        for s, (m, n, w) in enumerate(lay.dims):
            if w == 0:
                continue
            mp = maps[s]
            ov, ow, ob = int(lay.o_vw[s]), int(lay.o_gw[s]), int(lay.o_gb[s])
            # through the wake map: columns of X (trailing edge, convected rows) and of G
            px = torch.einsum("irjk,jrs->isjk", pw[:, 3 * ov:3 * (ov + (w + 1) * (n + 1))].reshape(NB, w + 1, n + 1, 3),
                              ops.tensor(mp.wz))
            qg = torch.einsum("irj,jrs->isj", qw[:, ow:ow + w * n].reshape(NB, w, n), ops.tensor(mp.wg))
            te_b = zb_c[0] + 3 * (int(lay.o_vb[s]) + m * (n + 1))
            phi[:, te_b:te_b + 3 * (n + 1)] -= px[:, 0].reshape(NB, 3 * (n + 1))   # X row 0: the input's TE row
            phi[:, gbc[0] + ob + (m - 1) * n:gbc[0] + ob + m * n] -= qg[:, 0]      # G row 0: gamma_b TE row
            if mp.n_g > 1:
                phi[:, gwc[0] + ow:gwc[0] + ow + (mp.n_g - 1) * n] -= qg[:, 1:].reshape(NB, (mp.n_g - 1) * n)
            conv_parts.append(px[:, 1:].reshape(NB, 3 * n_conv[s]))
        if cols("u", "nu_w") is not None:
            c0, c1 = cols("u", "nu_w")
            phi[:, c0:c1] -= dt * pw                                      # nu_w moves the new wake itself
        if conv_parts:
            pw_conv = torch.cat(conv_parts, dim=1)                        # (NB, 3 NC) in conv-target order
    # convection of the wake rows of step n (into the X rows of step n+1)
    need_conv = pw_conv is not None and NC > 0 and (free or prescribed)
    if need_conv:
        if free:
            jc_gb = ops.zeros(3 * NC, lay.NB)
            jc_gw = ops.zeros(3 * NC, lay.NW)
            for s in range(S):
                ops.ring(jc_gb, int(lay.o_gb[s]), t_conv, None, tZb[s], K, RC)
                if Zw[s].shape[0] > 1:
                    ops.ring(jc_gw, int(lay.o_gw[s]), t_conv, None, tZw[s], K, RC)
            gbc, gwc = cols("x", "gamma_b"), cols("x", "gamma_w")
            phi[:, gbc[0]:gbc[1]] -= dt * (pw_conv @ jc_gb)
            phi[:, gwc[0]:gwc[1]] -= dt * (pw_conv @ jc_gw)
        if prescribed:
            # d zw1[r+1] / d zw0[r] = I + dt grad(U + V_conv) at the convected vertex
            gconv = _flow_grad(ff, conv_flat, t)
            if free:
                lats0 = list(zip(tZb, tgb)) + [(z, g) for z, g in zip(tZw, tgw) if z.shape[0] > 1]
                for a in range(3):
                    lam = np.zeros((NC, 3))
                    lam[:, a] = 1.0
                    gconv[:, a, :] += ops.vind_grad_t(t_conv, lats0, K, RC, ops.tensor(lam)).cpu().numpy()
            blk = np.eye(3)[None] + dt * gconv                               # (NC, 3, 3)
            zwc = cols("x", "zeta_w")
            tblk = ops.tensor(blk)
            # -P_w[:, conv cols of zw1] . blk on the zw0 columns of the same vertex
            src_cols = np.concatenate([3 * (int(lay.o_vw[s]) + np.arange(n_conv[s])) for s in range(S)])
            pc = pw_conv.reshape(NB, NC, 3)
            contrib = -torch.einsum("iva,vab->ivb", pc, tblk)              # (NB, NC, 3)
            idx = torch.as_tensor((zwc[0] + src_cols[:, None] + np.arange(3)[None, :]).ravel(), device=pw.device)
            phi.index_add_(1, idx, contrib.reshape(NB, 3 * NC))
            if free:
                jc_zw = ops.zeros(3 * NC, 3 * lay.NVW)
                jc_zb = ops.zeros(3 * NC, 3 * lay.NVB)
                for s in range(S):
                    if Zw[s].shape[0] > 1:
                        ops.vertex(jc_zw, 3 * int(lay.o_vw[s]), t_conv, None, tZw[s], tgw[s], K, RC)
                    ops.vertex(jc_zb, 3 * int(lay.o_vb[s]), t_conv, None, tZb[s], tgb[s], K, RC)
                zbs = cols("x", "zeta_b")
                phi[:, zwc[0]:zwc[1]] -= dt * (pw_conv @ jc_zw)
                phi[:, zbs[0]:zbs[1]] -= dt * (pw_conv @ jc_zb)
    if rows:
        r_, c_, v_ = (np.concatenate(a) for a in (rows, cl, vals))
        phi.index_put_((torch.as_tensor(r_, device=phi.device), torch.as_tensor(c_, device=phi.device)),
                       torch.as_tensor(v_, device=phi.device), accumulate=True)
    _mask(phi, lay, lists["gamma_b"])
    ops.solve_many(lu, piv, phi)                                          # dGamma_b = A^-1 dPhi

    # ---- next-state rows ------------------------------------------------------------------
    R_state = ops.zeros(lay.n_states, ncol)
    r0, r1 = lay.x["gamma_b"]
    R_state[r0:r1] = phi
    gbc, gwc = cols("x", "gamma_b"), cols("x", "gamma_w")
    gw_r = lay.x["gamma_w"][0]
    ones_r, ones_c, ones_v = [], [], []                                   # sparse entries of R_state
    for s, (m, n, w) in enumerate(lay.dims):
        if w == 0:
            continue
        ow, ob = int(lay.o_gw[s]), int(lay.o_gb[s])
        j_, r_, g_ = np.nonzero(maps[s].wg)                               # gamma_w1[r, j] <- G[g, j]
        ones_r.append(gw_r + ow + r_ * n + j_)
        ones_c.append(np.where(g_ == 0, gbc[0] + ob + (m - 1) * n + j_, gwc[0] + ow + (g_ - 1) * n + j_))
        ones_v.append(maps[s].wg[j_, r_, g_])
    if "gamma_b_nm1" in lay.x:
        q0 = lay.x["gamma_b_nm1"][0]
        ones_r.append(q0 + np.arange(NB))
        ones_c.append(gbc[0] + np.arange(NB))
        ones_v.append(np.ones(NB))
    if prescribed:
        zr = lay.x["zeta_w"][0]
        zwc, zbi = cols("x", "zeta_w"), cols("u", "zeta_b")
        blk = np.zeros((0, 3, 3))
        if NC:
            gconv = _flow_grad(ff, conv_flat, t)
            if free:
                lats0 = list(zip(tZb, tgb)) + [(z, g) for z, g in zip(tZw, tgw) if z.shape[0] > 1]
                for a in range(3):
                    lam = np.zeros((NC, 3))
                    lam[:, a] = 1.0
                    gconv[:, a, :] += ops.vind_grad_t(t_conv, lats0, K, RC, ops.tensor(lam)).cpu().numpy()
            blk = np.eye(3)[None] + dt * gconv                           # d X[conv] / d zeta_w0 per vertex
        for s, (m, n, w) in enumerate(lay.dims):
            ov = int(lay.o_vw[s])
            j_, r_, x_ = np.nonzero(maps[s].wz)                           # zeta_w1[r, j] <- X[x, j]
            wv = maps[s].wz[j_, r_, x_]
            te = x_ == 0                                                  # X row 0: the input's TE row
            for k in range(3):
                ones_r.append(zr + 3 * (ov + r_[te] * (n + 1) + j_[te]) + k)
                ones_c.append(zbi[0] + 3 * (int(lay.o_vb[s]) + m * (n + 1) + j_[te]) + k)
                ones_v.append(wv[te])
            cv = ~te                                                      # convected rows of step n
            tgt = o_conv[s] + (x_[cv] - 1) * (n + 1) + j_[cv]
            for k in range(3):
                for b in range(3):
                    ones_r.append(zr + 3 * (ov + r_[cv] * (n + 1) + j_[cv]) + k)
                    ones_c.append(zwc[0] + 3 * (ov + (x_[cv] - 1) * (n + 1) + j_[cv]) + b)
                    ones_v.append(wv[cv] * blk[tgt, k, b])
        if NC and free:
            # the free convection's dense terms, through the wake map
            dense = [(zwc, jc_zw)] + ([(gbc, jc_gb), (gwc, jc_gw)] if wt == "free" else [])
            for s, (m, n, w) in enumerate(lay.dims):
                if w == 0:
                    continue
                mp, ov = maps[s], int(lay.o_vw[s])
                wz = ops.tensor(mp.wz)
                for cc_, jc in dense:
                    part = jc[3 * int(o_conv[s]):3 * int(o_conv[s + 1])].reshape(mp.n_conv_rows, n + 1, 3, -1)
                    x_part = torch.cat([torch.zeros_like(part[:1]), part], dim=0)   # X row 0 does not convect
                    rows_ = torch.einsum("jrs,sjkc->rjkc", wz, x_part).reshape(3 * (w + 1) * (n + 1), -1)
                    R_state[zr + 3 * ov:zr + 3 * (ov + (w + 1) * (n + 1)), cc_[0]:cc_[1]] += dt * rows_
        if cols("u", "nu_w") is not None:
            c0, _ = cols("u", "nu_w")
            R_state.index_put_((torch.as_tensor(zr + np.arange(3 * lay.NVW), device=R_state.device),
                                torch.as_tensor(c0 + np.arange(3 * lay.NVW), device=R_state.device)),
                               ops.tensor(np.full(3 * lay.NVW, dt)), accumulate=True)
        zbr = lay.x["zeta_b"][0]
        ones_r.append(zbr + np.arange(3 * lay.NVB))
        ones_c.append(zbi[0] + np.arange(3 * lay.NVB))
        ones_v.append(np.ones(3 * lay.NVB))
    if ones_r:
        r_, c_, v_ = np.concatenate(ones_r), np.concatenate(ones_c), np.concatenate(ones_v)
        R_state.index_put_((torch.as_tensor(r_, device=R_state.device), torch.as_tensor(c_, device=R_state.device)),
                           ops.tensor(v_), accumulate=True)

    # ---- output rows ----------------------------------------------------------------------
    R_out = ops.zeros(lay.n_outputs, ncol)
    fs0 = lay.y["f_steady"][0]
    R_out[fs0:fs0 + 3 * lay.NVB] = _steady_force_rows(ops, lay, cfg, Zb, Zw, gb, gw, tZb, tZw, tgb, tgw, lists)
    if "f_unsteady" in lay.y:
        fu0 = lay.y["f_unsteady"][0]
        gbm = cols("x", "gamma_b_nm1")
        rr, cc, vv = [], [], []
        for s, (m, n, w) in enumerate(lay.dims):
            k_, l_ = np.meshgrid(np.arange(m), np.arange(n), indexing="ij")
            i = (int(lay.o_gb[s]) + k_ * n + l_).ravel()
            for dk in (0, 1):
                for dl in (0, 1):
                    v = (int(lay.o_vb[s]) + (k_ + dk) * (n + 1) + l_ + dl).ravel()
                    for b in range(3):
                        val = 0.25 * rho / dt * n_flat[i, b]   # split_to_vertex over both axes: a quarter each
                        rr += [fu0 + 3 * v + b, fu0 + 3 * v + b]
                        cc += [gbc[0] + i, gbm[0] + i]
                        vv += [val, -val]
        R_out.index_put_((torch.as_tensor(np.concatenate(rr), device=R_out.device),
                          torch.as_tensor(np.concatenate(cc), device=R_out.device)),
                         ops.tensor(np.concatenate(vv)), accumulate=True)
        # d f_unsteady / d zeta_b = rho Gamma_dot split(dn): Gamma_dot is zero at the
        # reference point (gamma_b_n = gamma_b_nm1 = the reference circulation)
    return R_state, R_out


def _mask(mat, lay, diff):
    """Zero the column blocks a residual does not differentiate."""
    keep = set(diff)
    for kind, blocks in (("x", lay.x_blocks), ("u", lay.u_blocks)):
        for name, _ in blocks:
            if f"{kind}:{name}" not in keep:
                c0, c1 = lay.col(kind, name)
                mat[:, c0:c1] = 0.0


def _steady_force_rows(ops, lay, cfg, Zb, Zw, gb, gw, tZb, tZw, tgb, tgw, lists):
    """d f_steady over [states | inputs]: f = rho g (v_rel x r) per filament, split to the
    vertices (aero/utils.py:126-223), v_rel from the linear model's cutoff kernel."""
    torch = ops.torch
    S = len(lay.dims)
    ff, t, rho = cfg["flowfield"], cfg["t"], cfg["rho"]
    FK, FRC = _lib.FJ_KERNEL_CUTOFF, cfg["force_r_cut"]
    prescribed = cfg["wake_type"] in ("prescribed", "free")
    ncol = lay.n_states + lay.n_inputs
    # filaments of every surface: start, end vertex (global), strength coefficients
    fa, fb, mids, rvec, gval = [], [], [], [], []
    gcoef = []   # list of (filament, column-in-gamma_b or -1-(gamma_w col), coefficient)
    nf = 0
    for s, (m, n, w) in enumerate(lay.dims):
        z = Zb[s]
        vb, ob, ow = int(lay.o_vb[s]), int(lay.o_gb[s]), int(lay.o_gw[s])
        G = gb[s]
        for k in range(m):          # chordwise (k,l)->(k+1,l), g = G[k,l] - G[k,l-1]
            for l in range(n + 1):
                fa.append(vb + k * (n + 1) + l)
                fb.append(vb + (k + 1) * (n + 1) + l)
                g = (G[k, l] if l < n else 0.0) - (G[k, l - 1] if l >= 1 else 0.0)
                if l < n:
                    gcoef.append((nf, ob + k * n + l, 1.0))
                if l >= 1:
                    gcoef.append((nf, ob + k * n + l - 1, -1.0))
                gval.append(g)
                nf += 1
        for k in range(m + 1):      # spanwise (k,l)->(k,l+1), g = G[k-1,l] - G[k,l] (- G_w[0,l] at the TE)
            for l in range(n):
                fa.append(vb + k * (n + 1) + l)
                fb.append(vb + k * (n + 1) + l + 1)
                g = (G[k - 1, l] if k >= 1 else 0.0) - (G[k, l] if k < m else 0.0)
                if k >= 1:
                    gcoef.append((nf, ob + (k - 1) * n + l, 1.0))
                if k < m:
                    gcoef.append((nf, ob + k * n + l, -1.0))
                if k == m and w > 0:
                    g -= gw[s][0, l]
                    gcoef.append((nf, -1 - (ow + l), -1.0))
                gval.append(g)
                nf += 1
    fa, fb = np.asarray(fa), np.asarray(fb)
    zflat = np.concatenate([z.reshape(-1, 3) for z in Zb])
    mid = 0.5 * (zflat[fa] + zflat[fb])
    rv = zflat[fb] - zflat[fa]
    gval = np.asarray(gval)
    tmid = ops.tensor(mid)
    wake_lats = [(z, g) for z, g in zip(tZw, tgw) if z.shape[0] > 1]
    lats = list(zip(tZb, tgb)) + wake_lats
    v = ff(mid, t) + ops.vind(tmid, lats, FK, FRC).cpu().numpy()          # v_rel at the reference
    grad = _flow_grad(ff, mid, t)
    for a in range(3):
        lam = np.zeros((nf, 3))
        lam[:, a] = 1.0
        grad[:, a, :] += ops.vind_grad_t(tmid, lats, FK, FRC, ops.tensor(lam)).cpu().numpy()
    # dv (velocity at the midpoints) per column, 3 rows per filament
    dv = ops.zeros(3 * nf, ncol)
    gbc, gwc = lay.col("x", "gamma_b"), lay.col("x", "gamma_w")
    for s in range(S):
        ops.ring(dv, gbc[0] + int(lay.o_gb[s]), tmid, None, tZb[s], FK, FRC)
        if Zw[s].shape[0] > 1:
            ops.ring(dv, gwc[0] + int(lay.o_gw[s]), tmid, None, tZw[s], FK, FRC)
    zbc = lay.col("u", "zeta_b")
    for s in range(S):
        ops.vertex(dv, zbc[0] + 3 * int(lay.o_vb[s]), tmid, None, tZb[s], tgb[s], FK, FRC)
    if prescribed:
        zwc = lay.col("x", "zeta_w")
        for s in range(S):
            if Zw[s].shape[0] > 1:
                ops.vertex(dv, zwc[0] + 3 * int(lay.o_vw[s]), tmid, None, tZw[s], tgw[s], FK, FRC)
    rows, cl, vals = [], [], []
    fi = np.arange(nf)
    for end in (fa, fb):
        for a in range(3):
            for b in range(3):
                # the midpoint moves with both ends: grad v . 0.5 d zeta
                rows.append(3 * fi + a)
                cl.append(zbc[0] + 3 * end + b)
                vals.append(0.5 * grad[:, a, b])
            # - 0.5 zeta_dot (relative velocity) and + 0.5 nu_b (bound upwash input)
            rows.append(3 * fi + a)
            cl.append(lay.col("u", "zeta_b_dot")[0] + 3 * end + a)
            vals.append(np.full(nf, -0.5))
            if lay.col("u", "nu_b") is not None:
                rows.append(3 * fi + a)
                cl.append(lay.col("u", "nu_b")[0] + 3 * end + a)
                vals.append(np.full(nf, 0.5))
    r_, c_, v_ = (np.concatenate(x) for x in (rows, cl, vals))
    dev = dv.device
    dv.index_put_((torch.as_tensor(r_, device=dev), torch.as_tensor(c_, device=dev)), torch.as_tensor(v_, device=dev),
                  accumulate=True)
    # per filament: rho g (dv x r) + rho g (v x dr) + rho dg (v x r)
    dv3 = dv.reshape(nf, 3, ncol)
    r_t = ops.tensor(rv)[:, :, None].expand(nf, 3, ncol)
    df = torch.linalg.cross(dv3, r_t, dim=1)
    del dv, dv3, r_t
    df *= ops.tensor(rho * gval)[:, None, None]
    rows, cl, vals = [], [], []
    vx = _skew(v) * (rho * gval)[:, None, None]                           # rho g [v]x
    for sign, end in ((1.0, fb), (-1.0, fa)):
        for a in range(3):
            for b in range(3):
                rows.append(3 * fi + a)
                cl.append(zbc[0] + 3 * end + b)
                vals.append(sign * vx[:, a, b])
    vxr = rho * np.cross(v, rv)                                           # rho (v x r)
    for f, col, coef in gcoef:
        colg = gbc[0] + col if col >= 0 else gwc[0] + (-1 - col)
        for a in range(3):
            rows.append([3 * f + a])
            cl.append([colg])
            vals.append([coef * vxr[f, a]])
    r_, c_, v_ = (np.concatenate([np.ravel(x) for x in y]) for y in (rows, cl, vals))
    df = df.reshape(3 * nf, ncol)
    df.index_put_((torch.as_tensor(r_, device=dev), torch.as_tensor(c_, device=dev)), torch.as_tensor(v_, device=dev),
                  accumulate=True)
    # split to the vertices: each filament's force half to either end
    out = ops.zeros(3 * lay.NVB, ncol)
    df *= 0.5
    for end in (fa, fb):
        idx = torch.as_tensor((3 * end[:, None] + np.arange(3)[None, :]).ravel(), device=dev)
        out.index_add_(0, idx, df)
    del df
    _mask(out, lay, lists["f_steady"])
    return out


def _input_jacobians(proj: LinearInputProjection, nz: int):
    """(d zeta_b / d q, d zeta_b_dot / d q), each (nz, len q), of an input projection."""
    sizes = [int(v) for v in proj.arg_sizes]
    if len(proj.arg_names) != len(sizes) or len(proj.arg_refs) != len(sizes):
        raise ValueError("input projection: arg_names, arg_sizes and arg_refs must have the same length")
    q0 = np.concatenate([np.ravel(np.asarray(r, np.float64)) for r in proj.arg_refs])
    if q0.size != sum(sizes):
        raise ValueError(f"input projection: arg_refs hold {q0.size} values, arg_sizes sum to {sum(sizes)}")
    offs = np.concatenate([[0], np.cumsum(sizes)])

    def split(q):
        return {n: q[offs[i]:offs[i + 1]] for i, n in enumerate(proj.arg_names)}

    if proj.jacobian is not None:
        jzb, jzbd = (np.asarray(j, np.float64) for j in proj.jacobian(**split(q0)))
    else:
        jzb, jzbd = _fd_columns(lambda q: proj.to_zeta(**split(q)), q0, proj.fd_step)
    if jzb.shape != (nz, q0.size) or jzbd.shape != (nz, q0.size):
        raise ValueError(f"input projection: Jacobians must be ({nz}, {q0.size}), got {jzb.shape}, {jzbd.shape}")
    return jzb, jzbd


def _output_jacobians(proj: LinearOutputProjection, fs0, fu0):
    """(d out / d f_steady, d out / d f_unsteady or None) of an output projection at the
    reference forces fs0, fu0 (fu0 None without the unsteady force)."""
    if proj.jacobian is not None:
        jfs, jfu = proj.jacobian(fs0, fu0)
        jfs = np.asarray(jfs, np.float64)
        jfu = None if jfu is None else np.asarray(jfu, np.float64)
    else:
        n = fs0.size
        if fu0 is None:
            (jfs,) = _fd_columns(lambda f: (proj.to_output(f, None),), fs0, proj.fd_step)
            jfu = None
        else:
            (j,) = _fd_columns(lambda f: (proj.to_output(f[:n], f[n:]),), np.concatenate([fs0, fu0]), proj.fd_step)
            jfs, jfu = j[:, :n], j[:, n:]
    if jfs.shape != (int(proj.size), fs0.size):
        raise ValueError(f"output projection: Jacobian must be ({proj.size}, {fs0.size}), got {jfs.shape}")
    return jfs, jfu


def _project(torch, lay, a, b, c, d, jin=None, jout=None):
    """The reference's projections (:631-725) applied to the unprojected A, B, C, D.

    Input (jin = (J_zeta_b, J_zeta_b_dot)): the inputs become [q, nu_b, nu_w]; every
    derivative with respect to zeta_b and zeta_b_dot of step n+1 chains through J, and so
    does the bound circulation's derivative with respect to zeta_b of step n (a state of
    the prescribed and free wake types, which the projection also sets); those state
    columns of A become zero.  Output (jout = (J_f_steady, J_f_unsteady)): the outputs
    become J_fs f_steady + J_fu f_unsteady."""
    if jin is not None:
        jzb, jzbd = jin
        zb, zbd = lay.u["zeta_b"], lay.u["zeta_b_dot"]

        def project(m_state, m_in):
            q = m_in[:, zb[0]:zb[1]] @ jzb + m_in[:, zbd[0]:zbd[1]] @ jzbd
            if "zeta_b" in lay.x:
                z0, z1 = lay.x["zeta_b"]
                q = q + m_state[:, z0:z1] @ jzb
                m_state[:, z0:z1] = 0.0
            rest = [m_in[:, lay.u[k][0]:lay.u[k][1]] for k in ("nu_b", "nu_w") if k in lay.u]
            return torch.cat([q, *rest], dim=1)

        a, c = a.clone(), c.clone()
        b = project(a, b)
        d = project(c, d)
    if jout is not None:
        jfs, jfu = jout
        fs, fu = lay.y["f_steady"], lay.y.get("f_unsteady")
        c_new, d_new = jfs @ c[fs[0]:fs[1]], jfs @ d[fs[0]:fs[1]]
        if fu is not None and jfu is not None:
            c_new = c_new + jfu @ c[fu[0]:fu[1]]
            d_new = d_new + jfu @ d[fu[0]:fu[1]]
        c, d = c_new, d_new
    return a, b, c, d


# ---------------------------------------------------------------------------------------
# the public class
# ---------------------------------------------------------------------------------------
class LinearUVLM:
    """Linearised UVLM about a steady reference solution (aero/linear/linear_uvlm.py:81-).

    ``LinearUVLM(uvlm, reference, wake_type)`` with ``reference`` the snapshot of
    ``uvlm.solve_static()``; ``.sys`` is the ``LinearSystem`` (A, B, C, D on the device),
    ``.run(u, x0)`` marches it over input perturbations and returns the totals."""

    def __init__(self, case, reference, wake_type: str = "frozen", bound_upwash: bool = True,
                 wake_upwash: bool = True, unsteady_force: bool = True, *, skip_checks: bool = False,
                 skip_linearisation: bool = False, device=None):
        if wake_type not in WAKE_TYPES:
            raise ValueError(f"wake_type must be one of {WAKE_TYPES}, got {wake_type!r}")
        if case.kernel.kernel_id not in (_lib.FJ_KERNEL_EPSILON, _lib.FJ_KERNEL_CUTOFF):
            raise NotImplementedError("the linearisation is written for the epsilon and cutoff kernels")
        if any(p is not None for p in case.polars):
            raise NotImplementedError("polar corrections are not part of the linear model")
        self.case = case
        self.wake_type = wake_type
        self.prescribed_wake, self.free_wake = {"frozen": (False, False), "prescribed": (True, False),
                                                "free": (True, True)}[wake_type]
        self.bound_upwash, self.wake_upwash, self.unsteady_force = bound_upwash, wake_upwash, unsteady_force
        self.dt = float(case.dt)
        self._reference = reference
        g = lambda name: [np.asarray(a, np.float64) for a in getattr(reference, name)]
        self._ref = {"zeta_b": g("zeta_b"), "zeta_w": g("zeta_w"), "gamma_b": g("gamma_b"), "gamma_w": g("gamma_w"),
                     "zeta_b_dot": g("zeta_b_dot"), "f_steady": g("f_steady")}
        gbd = getattr(reference, "gamma_b_dot", None)
        self._ref["gamma_b_dot"] = ([np.zeros_like(a) for a in self._ref["gamma_b"]] if gbd is None else
                                    [np.asarray(a, np.float64) for a in gbd])
        fu = getattr(reference, "f_unsteady", None)
        self._ref["f_unsteady"] = ([np.zeros_like(a) for a in self._ref["f_steady"]] if fu is None else
                                   [np.asarray(a, np.float64) for a in fu])
        if not skip_checks:
            if max(np.abs(z).max() for z in self._ref["zeta_b_dot"]) > 1e-6:
                warnings.warn("Reference bound surface velocities are non-zero. Ensure that the reference state is "
                              "steady for linearisation.")
            if max(np.abs(z).max() for z in self._ref["gamma_b_dot"]) > 1e-6:
                warnings.warn("Reference bound circulation time derivative is non-zero. Ensure that the reference "
                              "state is steady for linearisation.")
        dims = [(gd.m, gd.n, gd.m_star) for gd in case.grid_disc]
        self.layout = _Layout(dims, wake_type, bound_upwash, wake_upwash, unsteady_force)
        self.n_inputs, self.n_states, self.n_outputs = (self.layout.n_inputs, self.layout.n_states,
                                                        self.layout.n_outputs)
        mirror = None if case.mirror_point is None else (case.mirror_point, case.mirror_normal)
        self._ops = _CudaOps(device, mirror)
        self._sys = None
        if not skip_linearisation:
            self._sys = self.linearise()

    @property
    def sys(self) -> LinearSystem:
        if self._sys is None:
            raise ValueError("System not linearised")
        return self._sys

    @property
    def reference(self):
        return self._reference

    def _config(self):
        kid = self.case.kernel.kernel_id
        return {"wake_type": self.wake_type, "free_wake": bool(self.case.free_wake), "kernel": kid,
                "r_cut": self.case.kernel.r_cut,
                # the linear model's force kernel is the cutoff kernel at the module radius
                # (aero/utils.py:648), the UVLM's own radius when it uses the cutoff kernel
                "force_r_cut": self.case.kernel.r_cut if kid == _lib.FJ_KERNEL_CUTOFF else R_CUTOFF,
                "dt": self.dt, "rho": self.case.flowfield.rho, "flowfield": self.case.flowfield,
                "t": float(np.asarray(self._reference.t).ravel()[0]), "bound_upwash": self.bound_upwash,
                "wake_upwash": self.wake_upwash, "unsteady_force": self.unsteady_force,
                "delta_w": [None if d is None else np.asarray(d, np.float64) for d in (self.case.delta_w or [])]
                or None}

    def linearise(self, batch_size=None, *, input_projection: LinearInputProjection | None = None,
                  output_projection: LinearOutputProjection | None = None) -> LinearSystem:
        """A, B, C, D about the reference (:727-829).  With an input projection the inputs
        are [projected arguments, nu_b, nu_w]: every residual's derivatives with respect to
        zeta_b and zeta_b_dot of step n+1 (and, for the bound circulation of the prescribed
        and free wake types, zeta_b of step n, which the projection also sets) chain
        through the projection's Jacobian, and the zeta_b state columns of A are zero
        (:631-698).  With an output projection the outputs are the projected forces
        (:700-725).  ``batch_size`` is accepted for the reference's signature."""
        lay = self.layout
        r_state, r_out = _assemble(self._ops, lay, self._ref, self._config())
        ns = lay.n_states
        jin = jout = None
        if input_projection is not None:
            jin = tuple(self._ops.tensor(j) for j in _input_jacobians(input_projection, 3 * lay.NVB))
        if output_projection is not None:
            fs0 = np.concatenate([np.ravel(x) for x in self._ref["f_steady"]])
            fu0 = np.concatenate([np.ravel(x) for x in self._ref["f_unsteady"]]) if self.unsteady_force else None
            jout = tuple(None if j is None else self._ops.tensor(j)
                         for j in _output_jacobians(output_projection, fs0, fu0))
        a, b, c, d = _project(self._ops.torch, lay, r_state[:, :ns], r_state[:, ns:], r_out[:, :ns], r_out[:, ns:],
                              jin, jout)
        # A | B and C | D stay views of the two assembled blocks (row stride n_states +
        # n_inputs): the products take strided operands, and no second copy is made
        return LinearSystem(a, b, c, d, self.dt)

    # -- vectors ------------------------------------------------------------------------
    def reference_states(self) -> np.ndarray:
        r = self._ref
        d = {"gamma_b": r["gamma_b"], "gamma_w": r["gamma_w"], "gamma_b_nm1": r["gamma_b"], "zeta_w": r["zeta_w"],
             "zeta_b": r["zeta_b"]}
        return np.concatenate([np.concatenate([np.ravel(a) for a in d[k]]) for k, _ in self.layout.x_blocks])

    def reference_outputs(self) -> np.ndarray:
        r = self._ref
        return np.concatenate([np.concatenate([np.ravel(a) for a in r[k]]) for k, _ in self.layout.y_blocks])

    def run_vectors(self, u, x0=None):
        """The linear system over packed input perturbations u (n_tstep, n_inputs) from the
        packed state perturbation x0: (x, y, x_total, y_total) as numpy arrays."""
        x, y = self.sys.run(u, x0)
        x, y = x.cpu().numpy(), y.cpu().numpy()
        return x, y, x + self.reference_states()[None], y + self.reference_outputs()[None]

    def _blocks_t(self, blocks, vec_t):
        """(n_tstep, size) -> {name: [per surface (n_tstep, *shape)]} in the blocks' order."""
        out, off = {}, 0
        n_t = vec_t.shape[0]
        for name, _ in blocks:
            tmpl = self._template(name)
            out[name] = []
            for a in tmpl:
                out[name].append(vec_t[:, off:off + a.size].reshape((n_t,) + a.shape))
                off += a.size
        return out

    def _template(self, name):
        r = self._ref
        return {"zeta_b": r["zeta_b"], "zeta_b_dot": r["zeta_b"], "nu_b": r["zeta_b"], "nu_w": r["zeta_w"],
                "gamma_b": r["gamma_b"], "gamma_w": r["gamma_w"], "gamma_b_nm1": r["gamma_b"],
                "zeta_w": r["zeta_w"], "f_steady": r["f_steady"], "f_unsteady": r["f_steady"]}[name]

    def _reference_value(self, name):
        r = self._ref
        if name in ("nu_b", "nu_w"):
            return [np.zeros_like(a) for a in self._template(name)]
        key = {"gamma_b_nm1": "gamma_b"}.get(name, name)
        return r[key]

    def run(self, u: AeroInputUnflattened, x0: AeroStateUnflattened | None = None, flowfield=None):
        """aero/linear/linear_uvlm.py:869-972: march the linear system over the input
        perturbations u (per surface, time-batched), from the state perturbation x0 (zero
        if None).  A flow field adds the bound and wake upwash perturbations
        U(zeta, t) - U(zeta, t_0) at the reference lattices, t = t_ref + i dt."""
        if self.prescribed_wake and self.sys.removed_u_np1:
            warnings.warn("Wake perturbations coordinates at the trailing edge are zero when removing u_np1 from the "
                          "system.")
        n_t = int(np.shape(u.zeta_b[0])[0])
        t0 = float(np.asarray(self._reference.t).ravel()[0])
        t = t0 + np.arange(n_t) * self.dt
        nu = {"nu_b": None if u.nu_b is None else [np.asarray(a, np.float64) for a in u.nu_b],
              "nu_w": None if u.nu_w is None else [np.asarray(a, np.float64) for a in u.nu_w]}
        for name, flag, lat in (("nu_b", self.bound_upwash, self._ref["zeta_b"]),
                                ("nu_w", self.wake_upwash, self._ref["zeta_w"])):
            if not flag:
                continue
            if flowfield is None and nu[name] is None:
                warnings.warn(f"No flowfield or {'bound' if name == 'nu_b' else 'wake'} upwash perturbations provided. "
                              f"Assuming zero {'bound' if name == 'nu_b' else 'wake'} upwash perturbations.")
                nu[name] = [np.zeros((n_t,) + z.shape) for z in lat]
            if flowfield is not None:
                flow = [np.stack([flowfield(z, ti) - flowfield(z, t[0]) for ti in t]) for z in lat]
                nu[name] = flow if nu[name] is None else [a + b for a, b in zip(nu[name], flow)]
        given = {"zeta_b": u.zeta_b, "zeta_b_dot": u.zeta_b_dot, **nu}
        u_vec = np.concatenate([np.concatenate([np.asarray(a, np.float64).reshape(n_t, -1) for a in given[k]], axis=1)
                                for k, _ in self.layout.u_blocks], axis=1)
        x0_vec = None
        if x0 is not None:
            x0_vec = np.concatenate([np.concatenate([np.ravel(a) for a in getattr(x0, k)])
                                     for k, _ in self.layout.x_blocks])
        x, y, _, _ = self.run_vectors(u_vec, x0_vec)
        ud = self._blocks_t(self.layout.u_blocks, u_vec)
        xd = self._blocks_t(self.layout.x_blocks, x)
        yd = self._blocks_t(self.layout.y_blocks, y)

        def total(d):
            return {k: [a + r[None] for a, r in zip(v, self._reference_value(k))] for k, v in d.items()}

        return AeroLinearResult(reference=self._reference, u_t=AeroInputUnflattened(**ud),
                                x_t=AeroStateUnflattened(**xd), y_t=AeroOutputUnflattened(**yd),
                                u_t_tot=AeroInputUnflattened(**total(ud)), x_t_tot=AeroStateUnflattened(**total(xd)),
                                y_t_tot=AeroOutputUnflattened(**total(yd)), n_tstep=n_t,
                                n_surf=len(self.layout.dims), t=t)
