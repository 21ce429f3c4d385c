"""Discrete adjoint of a prescribed-motion UVLM run (FP64).

Gradient of ``J = sum_n Fbar_n . F_n`` (F_n: total aerodynamic force of slot n, the sum
of ``f_steady + f_unsteady`` over vertices; e.g. time-averaged CL or CD) with respect to
the local lattice ``zeta_b0`` (and from there any shape parameter such as twist).  The
reference obtains the same gradient by reverse-mode AD through
``UVLM.solve_prescribed_dynamic`` (aero/uvlm.py:1335-1406).

Reverse step n (slot n back to n-1), with cotangents of circulations (Gb, Gw, Gdot),
wake geometry (Zw) and lattice (Zb, Zbdot):
  1. forces (aero/utils.py:126-223, uvlm.py:1093-1103): filament strength, relative
     velocity and filament vector terms; the induced velocity at the filament midpoints
     through the hand-written Biot-Savart VJP (``fj_vind_vjp``);
  2. gamma_dot filter (uvlm.py:691-715);
  3. solve: mu = A_n^-T Gb_n (``fj_lu_solve_t`` on the getrf factors of A_n that the
     forward recomputation of the segment kept, ``fj_case_factors_copy``);
  4. right-hand side and AIC: A_n Gamma_n = nc . V_bound(c), so the AIC's geometric
     derivative is the VJP of the bound-lattice sum at the collocation points; with the
     wake term both are one VJP with cotangent -mu nc;
  5. collocation points, normals, c_dot -> lattice vertices;
  6. wake shedding transposes (aero/utils.py:427-450): row r of wake n is row r-1 of
     wake n-1 (+ dt U), row 0 is the trailing edge of lattice n / TE circulation of n-1;
  7. node frames: zeta_b = R zeta_b0 + t, zeta_b_dot = Rdot zeta_b0 + tdot.
Slot 0 (the static solve, uvlm.py:1286-1333) closes the sweep with the lumped-wake AIC.

Forward states are recomputed from checkpoints every ``checkpoint`` steps (only the
checkpoint slots are kept), so device memory is O(checkpoint) slots and O(checkpoint)
factor matrices.

Scope: one surface (with or without a mirror image), epsilon or cutoff kernel, Constant
flow, prescribed or free wake (uniform or variable, ``delta_w``, with gradients through
the arc-length re-discretisation).  The free wake adds, per step, the VJP of its convection
velocity V(zeta_w_{n-1}; bound and wake of n-1): targets, both source lattices, both
circulations; the bound lattice's share is carried to the reverse step of slot n-1.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .runtime import device_of

FIELDS = ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
          "f_unsteady", "alpha")


class _Dev:
    """Device helpers around the C ABI (FP64)."""

    def __init__(self, device, kernel=None, r_cut=0.0, mirror=None):
        import torch

        self.torch = torch
        self.dev = device_of(device)
        self.kernel = _lib.FJ_KERNEL_EPSILON if kernel is None else kernel
        self.r_cut = float(r_cut)
        # image system across the plane (point, unit normal): host arrays for the C ABI
        self._mir = None if mirror is None else tuple(
            (C.c_double * 3)(*np.asarray(v, dtype=np.float64).tolist()) for v in mirror)
        self._ws = {}

    def t(self, a):
        return self.torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(self.dev)

    def ws(self, key, nbytes):
        w = self._ws.get(key)
        if w is None or w.numel() < nbytes:
            w = self.torch.empty(int(nbytes), dtype=self.torch.uint8, device=self.dev)
            self._ws[key] = w
        return w

    def stream(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def _lat(self, lats):
        n = len(lats)
        zs = [self.t(z) for z, _ in lats]
        gs = [self.t(g) for _, g in lats]
        return (zs, gs, (C.c_void_p * n)(*[z.data_ptr() for z in zs]), (C.c_void_p * n)(*[g.data_ptr() for g in gs]),
                (C.c_int * n)(*[z.shape[0] - 1 for z, _ in lats]), (C.c_int * n)(*[z.shape[1] - 1 for z, _ in lats]))

    def vind(self, targets, lats):
        tt = self.t(targets.reshape(-1, 3))
        zs, gs, zp, gp, rows, cols = self._lat(lats)
        n = C.c_size_t()
        mir = int(self._mir is not None)
        mp, mn = self._mir if mir else (None, None)
        _lib.call("fj_vind_workspace_size", tt.shape[0], rows, cols, len(lats), mir, _lib.FJ_PREC_FP64, C.byref(n))
        ws = self.ws("vind", n.value)
        out = self.torch.empty_like(tt)
        _lib.call("fj_vind", tt.data_ptr(), tt.shape[0], zp, gp, rows, cols, len(lats), mp, mn,
                  self.kernel, self.r_cut, _lib.FJ_PREC_FP64, out.data_ptr(), ws.data_ptr(), ws.numel(),
                  self.stream())
        return out.cpu().numpy().reshape(targets.shape)

    def vjp(self, targets, lats, lam):
        """(targets_bar, [zeta_bar], [gamma_bar]) of lam . v_ind(targets; lats)."""
        tt = self.t(targets.reshape(-1, 3))
        tl = self.t(lam.reshape(-1, 3))
        zs, gs, zp, gp, rows, cols = self._lat(lats)
        tb = self.torch.zeros_like(tt)
        zb = [self.torch.zeros_like(z) for z in zs]
        gb = [self.torch.zeros_like(g) for g in gs]
        n = len(lats)
        zbp = (C.c_void_p * n)(*[z.data_ptr() for z in zb])
        gbp = (C.c_void_p * n)(*[g.data_ptr() for g in gb])
        nb = C.c_size_t()
        mir = int(self._mir is not None)
        mp, mn = self._mir if mir else (None, None)
        _lib.call("fj_vind_vjp_workspace_size", tt.shape[0], rows, cols, n, mir, C.byref(nb))
        ws = self.ws("vjp", nb.value)
        _lib.call("fj_vind_vjp", tt.data_ptr(), tt.shape[0], zp, gp, rows, cols, n, mp, mn,
                  self.kernel, self.r_cut, tl.data_ptr(), tb.data_ptr(), zbp, gbp, ws.data_ptr(), ws.numel(),
                  self.stream())
        return (tb.cpu().numpy().reshape(targets.shape), [z.cpu().numpy() for z in zb],
                [g.cpu().numpy() for g in gb])

    def solve_t_factors(self, lu, piv, rhs):
        """mu with A^T mu = rhs from stored getrf factors (device tensors)."""
        n = piv.numel()
        w = C.c_size_t()
        _lib.call("fj_lu_workspace_size", n, C.byref(w))
        wl = self.ws("lu", w.value)
        b = self.t(rhs.ravel())
        _lib.call("fj_lu_solve_t", lu.data_ptr(), n, piv.data_ptr(), b.data_ptr(), wl.data_ptr(), wl.numel(),
                  self.stream())
        return b.cpu().numpy().reshape(rhs.shape)

    def solve_pair(self, zetas_b, rhs, rhs_t):
        """(x, mu) with A x = rhs and A^T mu = rhs_t, A the dynamic AIC of the bound
        lattices zetas_b, from one factorisation."""
        k = len(zetas_b)
        ms = [z.shape[0] - 1 for z in zetas_b]
        ns = [z.shape[1] - 1 for z in zetas_b]
        nb = sum(m * n for m, n in zip(ms, ns))
        tz = [self.t(z) for z in zetas_b]
        zp = (C.c_void_p * k)(*[z.data_ptr() for z in tz])
        mm, nn = (C.c_int * k)(*ms), (C.c_int * k)(*ns)
        a = self.torch.empty((nb, nb), dtype=self.torch.float64, device=self.dev)
        w = C.c_size_t()
        _lib.call("fj_aic_workspace_size", mm, nn, k, C.byref(w))
        ws = self.ws("aic", w.value)
        s = self.stream()
        mp, mn = self._mir if self._mir is not None else (None, None)
        _lib.call("fj_aic_assemble", zp, mm, nn, k, None, (C.c_int * k)(*([0] * k)), mp, mn, self.kernel, self.r_cut,
                  a.data_ptr(), ws.data_ptr(), ws.numel(), s)
        piv = self.torch.empty(nb, dtype=self.torch.int32, device=self.dev)
        _lib.call("fj_lu_workspace_size", nb, C.byref(w))
        wl = self.ws("lu", w.value)
        _lib.call("fj_lu_factor", a.data_ptr(), nb, piv.data_ptr(), wl.data_ptr(), wl.numel(), s)
        x = self.t(np.ravel(rhs))
        _lib.call("fj_lu_solve", a.data_ptr(), nb, piv.data_ptr(), x.data_ptr(), wl.data_ptr(), wl.numel(), s)
        mu = self.t(np.ravel(rhs_t))
        _lib.call("fj_lu_solve_t", a.data_ptr(), nb, piv.data_ptr(), mu.data_ptr(), wl.data_ptr(), wl.numel(), s)
        return x.cpu().numpy(), mu.cpu().numpy()

    def solve_t(self, zetas_b, zetas_w_static, rhs):
        """mu with A^T mu = rhs (flat, all surfaces), A the AIC of the bound lattices
        zetas_b (with each surface's wake lumped onto its TE column when zetas_w_static is
        given: the static solve)."""
        k = len(zetas_b)
        ms = [z.shape[0] - 1 for z in zetas_b]
        ns = [z.shape[1] - 1 for z in zetas_b]
        nb = sum(m * n for m, n in zip(ms, ns))
        tz = [self.t(z) for z in zetas_b]
        zp = (C.c_void_p * k)(*[z.data_ptr() for z in tz])
        mm, nn = (C.c_int * k)(*ms), (C.c_int * k)(*ns)
        wp, mstar = None, (C.c_int * k)(*([0] * k))
        if zetas_w_static is not None:
            tw = [self.t(z) for z in zetas_w_static]
            wp = (C.c_void_p * k)(*[z.data_ptr() for z in tw])
            mstar = (C.c_int * k)(*[z.shape[0] - 1 for z in zetas_w_static])
        a = self.torch.empty((nb, nb), dtype=self.torch.float64, device=self.dev)
        w = C.c_size_t()
        _lib.call("fj_aic_workspace_size", mm, nn, k, C.byref(w))
        ws = self.ws("aic", w.value)
        s = self.stream()
        mp, mn = self._mir if self._mir is not None else (None, None)
        _lib.call("fj_aic_assemble", zp, mm, nn, k, wp, mstar, mp, mn, self.kernel, self.r_cut, a.data_ptr(),
                  ws.data_ptr(), ws.numel(), s)
        piv = self.torch.empty(nb, dtype=self.torch.int32, device=self.dev)
        _lib.call("fj_lu_workspace_size", nb, C.byref(w))
        wl = self.ws("lu", w.value)
        _lib.call("fj_lu_factor", a.data_ptr(), nb, piv.data_ptr(), wl.data_ptr(), wl.numel(), s)
        b = self.t(np.ravel(rhs))
        _lib.call("fj_lu_solve_t", a.data_ptr(), nb, piv.data_ptr(), b.data_ptr(), wl.data_ptr(), wl.numel(), s)
        return b.cpu().numpy().reshape(np.shape(rhs))


def _avg4_T(bar_c, shape):
    """Transpose of the panel-centre average (neighbour_average over both axes)."""
    out = np.zeros(shape)
    q = 0.25 * bar_c
    out[:-1, :-1] += q
    out[1:, :-1] += q
    out[:-1, 1:] += q
    out[1:, 1:] += q
    return out


def _normals_T(zeta, bar_nc):
    """Transpose of nc = (z11 - z00) x (z10 - z01) (aero/utils.py:96-105)."""
    d1 = zeta[1:, 1:] - zeta[:-1, :-1]
    d2 = zeta[1:, :-1] - zeta[:-1, 1:]
    b1 = np.cross(d2, bar_nc)
    b2 = np.cross(bar_nc, d1)
    out = np.zeros(zeta.shape)
    out[1:, 1:] += b1
    out[:-1, :-1] -= b1
    out[1:, :-1] += b2
    out[:-1, 1:] -= b2
    return out


def _interp_T(x, xp, fp, fbar):
    """Transpose of np.interp(x, xp, fp) per output (1-D xp increasing): returns
    (xp_bar, fp_bar).  fp may carry trailing component axes; fbar matches x's shape plus
    them.  Inside [xp[j], xp[j+1]): f = fp[j] + t (fp[j+1] - fp[j]), t = (x - xp[j]) / dx;
    beyond the last node f = fp[-1] (no xp dependence); x is constant."""
    xp_bar = np.zeros(xp.shape)
    fp_bar = np.zeros(fp.shape)
    last = xp.shape[0] - 1
    for q in range(x.shape[0]):
        xq = x[q]
        if not xq >= xp[0]:
            fp_bar[0] += fbar[q]
            continue
        if xq >= xp[last]:
            fp_bar[last] += fbar[q]
            continue
        j = int(np.searchsorted(xp, xq, side="right")) - 1
        dx = xp[j + 1] - xp[j]
        t = (xq - xp[j]) / dx
        fp_bar[j] += (1.0 - t) * fbar[q]
        fp_bar[j + 1] += t * fbar[q]
        tbar = np.sum(fbar[q] * (fp[j + 1] - fp[j]))
        xp_bar[j] += tbar * (-(1.0 - t) / dx)
        xp_bar[j + 1] += tbar * (-t / dx)
    return xp_bar, fp_bar


def _variable_wake_T(zw_nm1, te_n, gb_te_nm1, gw_nm1, dw, dt, U, Zw_bar, Gw_bar, v_conv=None):
    """Transpose of propagate_surf_wake with delta_w for a prescribed wake
    (aero/utils.py:427-491, gradients through the arc lengths as the reference's default
    linearise_variable_wake=False).  Returns the cotangents of zeta_w at n-1, of the
    trailing-edge vertex row at n, of the trailing-edge circulation row at n-1 and of
    gamma_w at n-1.  ``v_conv``: the free wake's induced velocity at zw_nm1 (its own VJP is
    the caller's), so that the arc lengths are those of the convected rows."""
    W1, n1, _ = zw_nm1.shape          # W + 1 vertex rows, n + 1 columns
    vel = U if v_conv is None else U + v_conv                  # free wake: + induced velocity
    X = np.concatenate([te_n[None], zw_nm1 + dt * vel], axis=0)  # (W + 2, n + 1, 3)
    G = np.concatenate([gb_te_nm1[None], gw_nm1], axis=0)      # (W + 1, n)
    seg = np.linalg.norm(X[1:] - X[:-1], axis=-1)              # (W + 1, n + 1)
    S = np.concatenate([np.zeros((1, n1)), np.cumsum(seg, axis=0)], axis=0)
    SG = 0.5 * (0.5 * (S[:-1, :-1] + S[1:, :-1]) + 0.5 * (S[:-1, 1:] + S[1:, 1:]))
    s_disc = np.concatenate([np.zeros(1), np.cumsum(dw)])
    sg_disc = 0.5 * (s_disc[:-1] + s_disc[1:])
    X_bar = np.zeros_like(X)
    S_bar = np.zeros_like(S)
    for j in range(n1):
        sb, xb = _interp_T(s_disc, S[:, j], X[:, j], Zw_bar[:, j])
        S_bar[:, j] += sb
        X_bar[:, j] += xb
    G_bar = np.zeros_like(G)
    SG_bar = np.zeros_like(SG)
    if G.shape[0] > 1 or Gw_bar.size:
        for j in range(G.shape[1]):
            sgb, gb = _interp_T(sg_disc, SG[:, j], G[:, j], Gw_bar[:, j])
            SG_bar[:, j] += sgb
            G_bar[:, j] += gb
    q = 0.25 * SG_bar
    S_bar[:-1, :-1] += q
    S_bar[1:, :-1] += q
    S_bar[:-1, 1:] += q
    S_bar[1:, 1:] += q
    # S_r = sum_{p <= r} |X_p - X_{p-1}|
    D_bar = np.cumsum(S_bar[::-1], axis=0)[::-1][1:]          # (W + 1, n + 1): sum_{r >= p} S_bar_r
    d = X[1:] - X[:-1]
    e = d / np.maximum(np.linalg.norm(d, axis=-1, keepdims=True), 1e-300)
    X_bar[1:] += D_bar[..., None] * e
    X_bar[:-1] -= D_bar[..., None] * e
    return X_bar[1:], X_bar[0], G_bar[0], G_bar[1:]


def _flow_T(ff, x, t, ubar):
    """x-cotangent of u = ff(x, t) (aero/flowfields.py:87-181).  Zero for a Constant
    field.  For the 1-cos gust u = a (A/2)(1 - cos(pi g / L)) on 0 < g < 2L, with
    g = (x - x0 - U t) . d (U t only with relative motion), so
    x_bar = (ubar . a) (A/2)(pi/L) sin(pi g / L) d inside the gust, 0 outside (the
    reference's jax.vjp through jnp.where differentiates the taken branch)."""
    x = np.asarray(x)
    if not hasattr(ff, "gust_length"):
        return np.zeros_like(x)
    d, a = ff.gust_travel_direction, ff.gust_amplitude_direction
    L, A = ff.gust_length, ff.gust_amplitude
    rel = x - ff.gust_x0
    if ff.relative_motion:
        rel = rel - ff.u_inf * t
    g = rel @ d
    inside = (g > 0) & (g < 2.0 * L)
    coef = np.where(inside, 0.5 * A * (np.pi / L) * np.sin(np.pi * g / L), 0.0) * (np.asarray(ubar) @ a)
    return coef[..., None] * d


def _frames_T(bar_zb, bar_zbd, hg, hgd, dof):
    """zeta_b0 cotangent of zeta_b = R zeta_b0 + t and zeta_b_dot = Rdot zeta_b0 + tdot."""
    R = hg[dof][:, :3, :3]          # (n+1, 3, 3) per spanwise vertex column
    out = np.einsum("jki,mjk->mji", R, bar_zb)
    if bar_zbd is not None and hgd is not None:
        Rd = hgd[dof][:, :3, :3]
        out += np.einsum("jki,mjk->mji", Rd, bar_zbd)
    return out


class PrescribedAdjoint:
    """Forward + reverse sweep for one FP64 UVLM case (flapjax_b200.UVLM)."""

    def __init__(self, uvlm, device=None):
        if uvlm.kernel.kernel_id not in (_lib.FJ_KERNEL_EPSILON, _lib.FJ_KERNEL_CUTOFF):
            raise NotImplementedError("the adjoint is written for the epsilon and cutoff kernels")
        if uvlm.precision != "fp64":
            raise NotImplementedError("the adjoint runs in FP64")
        if any(p is not None for p in getattr(uvlm, "polars", ())):
            raise NotImplementedError("the adjoint does not differentiate the polar correction")
        self.uv = uvlm
        mirror = None if uvlm.mirror_point is None else (uvlm.mirror_point, uvlm.mirror_normal)
        self.d = _Dev(device, uvlm.kernel.kernel_id, uvlm.kernel.r_cut, mirror)

    # -- forward with checkpoints ------------------------------------------------------
    def _static(self):
        return self.uv.solve_static()

    def _run_segment(self, init_case, hg_seg, hgd_seg, keep_factors=False):
        """Forward over one segment; with ``keep_factors`` also the factors of every
        step's AIC (device tensors, index = slot in the segment)."""
        uv = self.uv
        dc = uv.make_device_case(hg_seg.shape[0], hg_seg.shape[1])
        uv.load_initial(dc, init_case)
        dc.set_hg(hg_seg, hgd_seg)
        if not keep_factors:
            dc.solve_dynamic(1, hg_seg.shape[0])
            return uv._to_case(dc)
        torch = self.d.torch
        nb = sum(g.m * g.n for g in uv.grid_disc)
        n = hg_seg.shape[0]
        lus = torch.empty((n, nb, nb), dtype=torch.float64, device=self.d.dev)
        pivs = torch.empty((n, nb), dtype=torch.int32, device=self.d.dev)
        for i in range(1, n):
            dc.solve_dynamic(i, i + 1)
            dc.copy_factors(lus[i], pivs[i])
        seg = uv._to_case(dc)
        seg.factors = (lus, pivs)
        return seg

    def gradient(self, hg_t, hg_dot_t, force_weights, checkpoint=10):
        """Return (J, dJ/dzeta_b0) for J = sum_{n>=1} force_weights[n] . F_n, F_n the total
        force on all surfaces at slot n; dJ/dzeta_b0 is an array for one surface and a
        list (one per surface) otherwise."""
        uv = self.uv
        hg_t = np.asarray(hg_t, float)
        hg_dot_t = np.asarray(hg_dot_t, float)
        fw = np.asarray(force_weights, float)
        N = hg_t.shape[0] - 1
        static = self._static()
        # forward: keep every checkpoint-th slot as a snapshot
        ckpt = {0: static}
        J = 0.0
        cur = static
        for s0 in range(0, N, checkpoint):
            s1 = min(N, s0 + checkpoint)
            seg = self._run_segment(cur, hg_t[s0:s1 + 1], hg_dot_t[s0:s1 + 1])
            for n in range(1, s1 - s0 + 1):
                J += float(fw[s0 + n] @ seg.force_total[n])
            cur = seg[s1 - s0]
            ckpt[s1] = cur
        # reverse: per surface, the cotangents of slot n's state flowing into step n
        dims = [(g.m, g.n, g.m_star) for g in uv.grid_disc]
        zeta0_bar = [np.zeros_like(np.asarray(z, float)) for z in uv.zeta_b0]
        Gb_next = [np.zeros((m, n)) for m, n, _ in dims]
        Gbd_next = [np.zeros((m, n)) for m, n, _ in dims]
        Gw_next = [np.zeros((W, n)) for _, n, W in dims]
        Zw_next = [np.zeros((W + 1, n + 1, 3)) for _, n, W in dims]
        Zb_next = [np.zeros((m + 1, n + 1, 3)) for m, n, _ in dims]  # free wake: from step n+1
        seg_starts = sorted(k for k in ckpt if k < N)
        for s0 in reversed(seg_starts):
            s1 = min(N, s0 + checkpoint)
            seg = self._run_segment(ckpt[s0], hg_t[s0:s1 + 1], hg_dot_t[s0:s1 + 1], keep_factors=True)
            for loc in range(s1 - s0, 0, -1):
                nstep = s0 + loc
                Gb_next, Gbd_next, Gw_next, Zw_next, Zb_next = self._reverse_step(
                    seg, loc, fw[nstep], Gb_next, Gbd_next, Gw_next, Zw_next, Zb_next, zeta0_bar, hg_t[nstep],
                    hg_dot_t[nstep])
        self._reverse_static(static, Gb_next, Gw_next, Zw_next, Zb_next, zeta0_bar, uv.hg_ref)
        return J, (zeta0_bar[0] if len(zeta0_bar) == 1 else zeta0_bar)

    # -- one dynamic reverse step ------------------------------------------------------
    def _reverse_step(self, seg, loc, Fbar, Gb_n, Gbd_n, Gw_n, Zw_n, Zb_n, zeta0_bar, hg_n, hgd_n):
        d, uv = self.d, self.uv
        ff = uv.flowfield
        dt, relax, rho = uv.dt, uv.gamma_dot_relaxation, ff.rho
        t_n = float(np.ravel(seg.t)[loc]) if np.ndim(seg.t) else float(seg.t)
        S = len(Gb_n)
        sl = range(S)
        zb = [seg.zeta_b[s][loc] for s in sl]
        zbd = [seg.zeta_b_dot[s][loc] for s in sl]
        zw = [seg.zeta_w[s][loc] for s in sl]
        gb = [seg.gamma_b[s][loc] for s in sl]
        gw = [seg.gamma_w[s][loc] for s in sl]
        gbd = [seg.gamma_b_dot[s][loc] for s in sl]
        nc = [seg.nc[s][loc] for s in sl]
        c = [seg.c[s][loc] for s in sl]
        Zb = [a.copy() for a in Zb_n]
        Zbd = [np.zeros_like(a) for a in zbd]
        Gb = [a.copy() for a in Gb_n]
        Gw = [a.copy() for a in Gw_n]
        Zw = [a.copy() for a in Zw_n]
        Gbd = [a.copy() for a in Gbd_n]
        lats = [(zw[s], gw[s]) for s in sl] + [(zb[s], gb[s]) for s in sl]  # lattice i: wake i, bound S + i
        # 1. forces: f = rho Gamma_eff (v_rel x r) per filament, v_rel = u + V - zeta_dot (midpoints)
        mp_c = [0.5 * (z[:-1] + z[1:]) for z in zb]
        mp_s = [0.5 * (z[:, :-1] + z[:, 1:]) for z in zb]
        parts = []
        for s in sl:
            parts += [mp_c[s].reshape(-1, 3), mp_s[s].reshape(-1, 3)]
        sizes = [p.shape[0] for p in parts]
        offs = np.concatenate([[0], np.cumsum(sizes)])
        targets = np.concatenate(parts)
        v = d.vind(targets, lats)
        lam = np.zeros_like(targets)
        vbar = []
        for s in sl:
            m, n_ = gb[s].shape
            v_c = v[offs[2 * s]:offs[2 * s + 1]].reshape(mp_c[s].shape)
            v_s = v[offs[2 * s + 1]:offs[2 * s + 2]].reshape(mp_s[s].shape)
            mpd_c = 0.5 * (zbd[s][:-1] + zbd[s][1:])
            mpd_s = 0.5 * (zbd[s][:, :-1] + zbd[s][:, 1:])
            vr_c, vr_s = ff(mp_c[s], t_n) + v_c - mpd_c, ff(mp_s[s], t_n) + v_s - mpd_s
            g_c = np.zeros((m, n_ + 1))
            g_c[:, :-1] = gb[s]
            g_c[:, 1:] += -gb[s]
            g_s = np.zeros((m + 1, n_))
            g_s[:-1, :] = -gb[s]
            g_s[1:, :] += gb[s]
            if gw[s].shape[0] > 0:
                g_s[-1, :] += -gw[s][0, :]
            r_c = zb[s][1:] - zb[s][:-1]
            r_s = zb[s][:, 1:] - zb[s][:, :-1]
            gbar_c = rho * np.einsum("ijk,k->ij", np.cross(vr_c, r_c), Fbar)
            gbar_s = rho * np.einsum("ijk,k->ij", np.cross(vr_s, r_s), Fbar)
            vbar_c = rho * g_c[..., None] * np.cross(r_c, Fbar)
            vbar_s = rho * g_s[..., None] * np.cross(r_s, Fbar)
            rbar_c = rho * g_c[..., None] * np.cross(Fbar, vr_c)
            rbar_s = rho * g_s[..., None] * np.cross(Fbar, vr_s)
            Zb[s][1:] += rbar_c
            Zb[s][:-1] -= rbar_c
            Zb[s][:, 1:] += rbar_s
            Zb[s][:, :-1] -= rbar_s
            Zbd[s][:-1] += -0.5 * vbar_c
            Zbd[s][1:] += -0.5 * vbar_c
            Zbd[s][:, :-1] += -0.5 * vbar_s
            Zbd[s][:, 1:] += -0.5 * vbar_s
            Gb[s] += gbar_c[:, :-1]      # g_c[k,l] = G[k,l] (l < n) - G[k,l-1] (l >= 1)
            Gb[s] -= gbar_c[:, 1:]
            Gb[s] -= gbar_s[:-1, :]      # g_s[k,l] = -G[k,l] (k < m) + G[k-1,l] (k >= 1)
            Gb[s] += gbar_s[1:, :]
            if gw[s].shape[0] > 0:
                Gw[s][0, :] -= gbar_s[-1, :]
            lam[offs[2 * s]:offs[2 * s + 1]] = vbar_c.reshape(-1, 3)
            lam[offs[2 * s + 1]:offs[2 * s + 2]] = vbar_s.reshape(-1, 3)
            vbar.append((vbar_c, vbar_s))
        tbar, zbar, gbars = d.vjp(targets, lats, lam)
        for s in sl:
            mpbar_c = tbar[offs[2 * s]:offs[2 * s + 1]].reshape(mp_c[s].shape) + _flow_T(ff, mp_c[s], t_n, vbar[s][0])
            mpbar_s = tbar[offs[2 * s + 1]:offs[2 * s + 2]].reshape(mp_s[s].shape) + _flow_T(ff, mp_s[s], t_n,
                                                                                            vbar[s][1])
            Zb[s][:-1] += 0.5 * mpbar_c
            Zb[s][1:] += 0.5 * mpbar_c
            Zb[s][:, :-1] += 0.5 * mpbar_s
            Zb[s][:, 1:] += 0.5 * mpbar_s
            Zw[s] += zbar[s]
            Zb[s] += zbar[S + s]
            Gw[s] += gbars[s]
            Gb[s] += gbars[S + s]
        # unsteady force rho * gamma_dot * nc; 2. gamma_dot filter
        ncbar, Gb_prev, Gbd_prev = [], [], []
        for s in sl:
            Gbd[s] += rho * np.einsum("ijk,k->ij", nc[s], Fbar)
            ncbar.append(rho * gbd[s][..., None] * Fbar)
            Gb[s] += (relax / dt) * Gbd[s]
            Gb_prev.append(-(relax / dt) * Gbd[s])
            Gbd_prev.append((1.0 - relax) * Gbd[s])
        # 3. transpose solve with A_n (all surfaces)
        rhs = np.concatenate([g.ravel() for g in Gb])
        factors = getattr(seg, "factors", None)
        mu_flat = (d.solve_t(zb, None, rhs) if factors is None
                   else d.solve_t_factors(factors[0][loc], factors[1][loc], rhs))
        po = np.concatenate([[0], np.cumsum([g.size for g in gb])])
        mu = [mu_flat[po[s]:po[s + 1]].reshape(gb[s].shape) for s in sl]
        # 4. RHS + AIC geometry: b = -(u - c_dot + V_w(c)) . nc and A Gamma = nc . V_b(c)
        cdot = [0.5 * (0.5 * (z[:-1, :-1] + z[1:, :-1]) + 0.5 * (z[:-1, 1:] + z[1:, 1:])) for z in zbd]
        co = np.concatenate([[0], np.cumsum([x.shape[0] * x.shape[1] for x in c])])
        c_all = np.concatenate([x.reshape(-1, 3) for x in c])
        Vtot = d.vind(c_all, lats)
        lam_c = [-mu[s][..., None] * nc[s] for s in sl]
        cdotbar = []
        for s in sl:
            Vs = Vtot[co[s]:co[s + 1]].reshape(c[s].shape)
            ncbar[s] += -mu[s][..., None] * (ff(c[s], t_n) - cdot[s] + Vs)
            cdotbar.append(mu[s][..., None] * nc[s])
        cbar_all, zbar2, gbar2 = d.vjp(c_all, lats, np.concatenate([x.reshape(-1, 3) for x in lam_c]))
        for s in sl:
            cbar = cbar_all[co[s]:co[s + 1]].reshape(c[s].shape) + _flow_T(ff, c[s], t_n, lam_c[s])
            Zw[s] += zbar2[s]
            Zb[s] += zbar2[S + s]
            Gw[s] += gbar2[s]   # the bound part belongs to the solve's linearity in Gamma
            # 5. geometry
            Zb[s] += _avg4_T(cbar, zb[s].shape)
            Zb[s] += _normals_T(zb[s], ncbar[s])
            Zbd[s] += _avg4_T(cdotbar[s], zbd[s].shape)
        # 6. wake shedding transposes; the free wake's convection velocity
        #    V(zw_{n-1}; all lattices of n-1) adds its own VJP
        zw_nm1 = [seg.zeta_w[s][loc - 1] for s in sl]
        gw_nm1 = [seg.gamma_w[s][loc - 1] for s in sl]
        zb_nm1 = [seg.zeta_b[s][loc - 1] for s in sl]
        gb_nm1 = [seg.gamma_b[s][loc - 1] for s in sl]
        lats_nm1 = [(zb_nm1[s], gb_nm1[s]) for s in sl] + [(zw_nm1[s], gw_nm1[s]) for s in sl]
        dws = getattr(uv, "delta_w", None) or [None] * S
        free = bool(uv.free_wake)
        Zw_prev, Gw_prev, Zb_prev = [], [], [np.zeros_like(z) for z in zb]
        conv = []  # per surface: (rows of zw_{n-1} convected, their cotangent)
        for s in sl:
            W = gw[s].shape[0]
            if dws[s] is not None:
                v_conv = d.vind(zw_nm1[s], lats_nm1) if (free and W > 0) else None
                zw_p, te_bar, gte_bar, gw_p = _variable_wake_T(
                    zw_nm1[s], zb[s][-1], gb_nm1[s][-1], gw_nm1[s], np.asarray(dws[s], float), dt,
                    ff(zw_nm1[s], t_n), Zw[s], Gw[s], v_conv)
                Zb[s][-1] += te_bar
                Zw_prev.append(zw_p)
                Gw_prev.append(gw_p)
                Gb_prev[s][-1, :] += gte_bar
                rows, cb = slice(None), np.array(zw_p)  # every row of zw_{n-1} is convected
            else:
                Zb[s][-1] += Zw[s][0]
                zp = np.zeros_like(Zw[s])
                zp[:-1] += Zw[s][1:]
                gp = np.zeros_like(Gw[s])
                if W > 0:
                    Gb_prev[s][-1, :] += Gw[s][0, :]
                    gp[:-1] += Gw[s][1:]
                Zw_prev.append(zp)
                Gw_prev.append(gp)
                rows, cb = slice(0, W), np.array(Zw[s][1:])
            # x_r = zw_{n-1,r} + dt (u(zw_{n-1,r}, t_n) + ...): the flow's own dependence on x
            Zw_prev[s][rows] += dt * _flow_T(ff, zw_nm1[s][rows], t_n, cb)
            conv.append((rows, cb))
        if free:
            tparts = [zw_nm1[s][conv[s][0]].reshape(-1, 3) for s in sl]
            lparts = [dt * conv[s][1].reshape(-1, 3) for s in sl]
            to = np.concatenate([[0], np.cumsum([p.shape[0] for p in tparts])])
            if to[-1] > 0:
                tbar, zbar_c, gbar_c = d.vjp(np.concatenate(tparts), lats_nm1, np.concatenate(lparts))
                for s in sl:
                    Zw_prev[s][conv[s][0]] += tbar[to[s]:to[s + 1]].reshape(zw_nm1[s][conv[s][0]].shape)
                    Zb_prev[s] += zbar_c[s]
                    Zw_prev[s] += zbar_c[S + s]
                    Gb_prev[s] += gbar_c[s]
                    Gw_prev[s] += gbar_c[S + s]
        # 7. node frames
        for s in sl:
            zeta0_bar[s] += _frames_T(Zb[s], Zbd[s], hg_n, hgd_n, uv.dof_mapping[s])
        return Gb_prev, Gbd_prev, Gw_prev, Zw_prev, Zb_prev

    def _reverse_static(self, st, Gb0, Gw0, Zw0, Zb0, zeta0_bar, hg0):
        d, uv = self.d, self.uv
        ff = uv.flowfield
        t0 = float(np.ravel(st.t)[0]) if np.ndim(st.t) else float(st.t)
        S = len(Gb0)
        sl = range(S)
        zb = [st.zeta_b[s] for s in sl]
        zw = [st.zeta_w[s] for s in sl]
        gb = [st.gamma_b[s] for s in sl]
        gw = [st.gamma_w[s] for s in sl]
        nc = [st.nc[s] for s in sl]
        c = [st.c[s] for s in sl]
        Gb = [g.copy() for g in Gb0]
        Zw = [z.copy() for z in Zw0]
        for s in sl:
            if Gw0[s].shape[0] > 0:
                Gb[s][-1, :] += Gw0[s].sum(axis=0)  # gamma_w = broadcast of the TE row (uvlm.py:995-1012)
        lumped = [z if g.shape[0] > 0 else None for z, g in zip(zw, Gw0)]
        rhs = np.concatenate([g.ravel() for g in Gb])
        mu_flat = d.solve_t(zb, None if all(x is None for x in lumped) else zw, rhs)
        po = np.concatenate([[0], np.cumsum([g.size for g in gb])])
        mu = [mu_flat[po[s]:po[s + 1]].reshape(gb[s].shape) for s in sl]
        lats = [(zw[s], gw[s]) for s in sl] + [(zb[s], gb[s]) for s in sl]
        co = np.concatenate([[0], np.cumsum([x.shape[0] * x.shape[1] for x in c])])
        c_all = np.concatenate([x.reshape(-1, 3) for x in c])
        Vtot = d.vind(c_all, lats)
        lam_c = [-mu[s][..., None] * nc[s] for s in sl]
        cbar_all, zbar, _ = d.vjp(c_all, lats, np.concatenate([x.reshape(-1, 3) for x in lam_c]))
        for s in sl:
            ncbar = -mu[s][..., None] * (ff(c[s], t0) + Vtot[co[s]:co[s + 1]].reshape(c[s].shape))
            cbar = cbar_all[co[s]:co[s + 1]].reshape(c[s].shape) + _flow_T(ff, c[s], t0, lam_c[s])
            Zw[s] += zbar[s]
            Zb = zbar[S + s] + Zb0[s]
            Zb[-1] += Zw[s].sum(axis=0)  # every wake row = TE + s_r u_dir (uvlm.py:662-689)
            Zb += _avg4_T(cbar, zb[s].shape)
            Zb += _normals_T(zb[s], ncbar)
            zeta0_bar[s] += _frames_T(Zb, None, hg0, None, uv.dof_mapping[s])


def twist_jacobian(m, n, chord, ea, ctrl_y, span_y, twist, camber=0.0):
    """d zeta_b0 / d theta for cases.twisted_grid with twist = interp(span_y, ctrl_y, theta):
    returns (n_ctrl, m+1, n+1, 3)."""
    from .cases import naca_camber

    xc = np.linspace(0.0, 1.0, m + 1)
    x = (xc - ea) * chord
    z = naca_camber(xc, camber) * chord if camber else np.zeros_like(xc)
    n_ctrl = len(ctrl_y)
    P = np.zeros((n + 1, n_ctrl))
    for k in range(n_ctrl):
        e = np.zeros(n_ctrl)
        e[k] = 1.0
        P[:, k] = np.interp(span_y, ctrl_y, e)
    dz = np.zeros((n + 1, m + 1, 3))
    for j in range(n + 1):
        c_, s_ = np.cos(twist[j]), np.sin(twist[j])
        dz[j, :, 0] = -s_ * x + c_ * z
        dz[j, :, 2] = -c_ * x - s_ * z
    return np.einsum("jk,jmd->kmjd", P, dz)
