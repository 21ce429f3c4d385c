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

    def solve_t(self, zeta_b, zeta_w_static, rhs):
        """mu with A^T mu = rhs, A the AIC of zeta_b (with the wake lumped onto the TE
        column when zeta_w_static is given: the static solve)."""
        m, n = zeta_b.shape[0] - 1, zeta_b.shape[1] - 1
        nb = m * n
        tz = self.t(zeta_b)
        zp = (C.c_void_p * 1)(tz.data_ptr())
        mm, nn = (C.c_int * 1)(m), (C.c_int * 1)(n)
        wp, ms = None, (C.c_int * 1)(0)
        if zeta_w_static is not None:
            tw = self.t(zeta_w_static)
            wp = (C.c_void_p * 1)(tw.data_ptr())
            ms = (C.c_int * 1)(zeta_w_static.shape[0] - 1)
        a = self.torch.empty((nb, nb), dtype=self.torch.float64, device=self.dev)
        w = C.c_size_t()
        _lib.call("fj_aic_workspace_size", mm, nn, 1, C.byref(w))
        ws = self.ws("aic", w.value)
        s = self.stream()
        mp, mn = self._mir if self._mir is not None else (None, None)
        _lib.call("fj_aic_assemble", zp, mm, nn, 1, wp, ms, mp, mn, self.kernel, self.r_cut, a.data_ptr(),
                  ws.data_ptr(), ws.numel(), s)
        piv = self.torch.empty(nb, dtype=self.torch.int32, device=self.dev)
        _lib.call("fj_lu_workspace_size", nb, C.byref(w))
        wl = self.ws("lu", w.value)
        _lib.call("fj_lu_factor", a.data_ptr(), nb, piv.data_ptr(), wl.data_ptr(), wl.numel(), s)
        b = self.t(rhs.ravel())
        _lib.call("fj_lu_solve_t", a.data_ptr(), nb, piv.data_ptr(), b.data_ptr(), wl.data_ptr(), wl.numel(), s)
        return b.cpu().numpy().reshape(rhs.shape)


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
        if uvlm.n_surf != 1:
            raise NotImplementedError("the adjoint handles one surface")
        if uvlm.kernel.kernel_id not in (_lib.FJ_KERNEL_EPSILON, _lib.FJ_KERNEL_CUTOFF):
            raise NotImplementedError("the adjoint is written for the epsilon and cutoff kernels")
        if uvlm.precision != "fp64":
            raise NotImplementedError("the adjoint runs in FP64")
        from .flowfields import Constant

        if not isinstance(uvlm.flowfield, Constant):
            raise NotImplementedError("the adjoint assumes a uniform (Constant) flow")
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
        """Return (J, dJ/dzeta_b0) for J = sum_{n>=1} force_weights[n] . F_n."""
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
        # reverse
        g = uv.grid_disc[0]
        m, n_, W = g.m, g.n, g.m_star
        dt, relax, rho = uv.dt, uv.gamma_dot_relaxation, uv.flowfield.rho
        U = uv.flowfield.u_inf
        dof = uv.dof_mapping[0]
        zeta0_bar = np.zeros_like(uv.zeta_b0[0])
        Gb_next = np.zeros((m, n_))      # cotangent of Gamma_b at slot n (being completed)
        Gbd_next = np.zeros((m, n_))
        Gw_next = np.zeros((W, n_))
        Zw_next = np.zeros((W + 1, n_ + 1, 3))
        Zb_next = np.zeros((m + 1, n_ + 1, 3))  # free wake: cotangent of slot n's lattice from step n+1
        seg_starts = sorted(k for k in ckpt if k < N)
        for s0 in reversed(seg_starts):
            s1 = min(N, s0 + checkpoint)
            seg = self._run_segment(ckpt[s0], hg_t[s0:s1 + 1], hg_dot_t[s0:s1 + 1], keep_factors=True)
            for loc in range(s1 - s0, 0, -1):
                nstep = s0 + loc
                Gb_next, Gbd_next, Gw_next, Zw_next, Zb_next = self._reverse_step(
                    seg, loc, fw[nstep], Gb_next, Gbd_next, Gw_next, Zw_next, Zb_next, zeta0_bar, hg_t[nstep],
                    hg_dot_t[nstep], dof, m, n_, W, dt, relax, rho, U)
        self._reverse_static(static, Gb_next, Gw_next, Zw_next, Zb_next, zeta0_bar, uv.hg_ref, dof, m, n_, W, U)
        return J, zeta0_bar

    # -- one dynamic reverse step ------------------------------------------------------
    def _reverse_step(self, seg, loc, Fbar, Gb_n, Gbd_n, Gw_n, Zw_n, Zb_n, zeta0_bar, hg_n, hgd_n, dof, m, n_, W,
                      dt, relax, rho, U):
        d = self.d
        zb = seg.zeta_b[0][loc]
        zbd = seg.zeta_b_dot[0][loc]
        zw = seg.zeta_w[0][loc]
        gb = seg.gamma_b[0][loc]
        gw = seg.gamma_w[0][loc]
        gbd = seg.gamma_b_dot[0][loc]
        nc = seg.nc[0][loc]
        c = seg.c[0][loc]
        Zb = Zb_n.copy()
        Zbd = np.zeros_like(zbd)
        Gb = Gb_n.copy()
        Gw = Gw_n.copy()
        Zw = Zw_n.copy()
        Gbd = Gbd_n.copy()
        # 1. forces
        mp_c = 0.5 * (zb[:-1] + zb[1:])
        mp_s = 0.5 * (zb[:, :-1] + zb[:, 1:])
        targets = np.concatenate([mp_c.reshape(-1, 3), mp_s.reshape(-1, 3)])
        lats = [(zw, gw), (zb, gb)]
        v = d.vind(targets, lats)
        nc_ = mp_c.shape[0] * mp_c.shape[1]
        v_c, v_s = v[:nc_].reshape(mp_c.shape), v[nc_:].reshape(mp_s.shape)
        mpd_c = 0.5 * (zbd[:-1] + zbd[1:])
        mpd_s = 0.5 * (zbd[:, :-1] + zbd[:, 1:])
        vr_c, vr_s = U + v_c - mpd_c, U + v_s - mpd_s
        g_c = np.zeros((m, n_ + 1))
        g_c[:, :-1] = gb
        g_c[:, 1:] += -gb
        g_s = np.zeros((m + 1, n_))
        g_s[:-1, :] = -gb
        g_s[1:, :] += gb
        if W > 0:
            g_s[-1, :] += -gw[0, :]
        r_c = zb[1:] - zb[:-1]
        r_s = zb[:, 1:] - zb[:, :-1]
        gbar_c = rho * np.einsum("ijk,k->ij", np.cross(vr_c, r_c), Fbar)
        gbar_s = rho * np.einsum("ijk,k->ij", np.cross(vr_s, r_s), Fbar)
        vbar_c = rho * g_c[..., None] * np.cross(r_c, Fbar)
        vbar_s = rho * g_s[..., None] * np.cross(r_s, Fbar)
        rbar_c = rho * g_c[..., None] * np.cross(Fbar, vr_c)
        rbar_s = rho * g_s[..., None] * np.cross(Fbar, vr_s)
        Zb[1:] += rbar_c
        Zb[:-1] -= rbar_c
        Zb[:, 1:] += rbar_s
        Zb[:, :-1] -= rbar_s
        Zbd[:-1] += -0.5 * vbar_c
        Zbd[1:] += -0.5 * vbar_c
        Zbd[:, :-1] += -0.5 * vbar_s
        Zbd[:, 1:] += -0.5 * vbar_s
        Gb += gbar_c[:, :-1]      # g_c[k,l] = G[k,l] (l < n) - G[k,l-1] (l >= 1)
        Gb -= gbar_c[:, 1:]
        Gb -= gbar_s[:-1, :]      # g_s[k,l] = -G[k,l] (k < m) + G[k-1,l] (k >= 1)
        Gb += gbar_s[1:, :]
        if W > 0:
            Gw[0, :] -= gbar_s[-1, :]
        lam = np.concatenate([vbar_c.reshape(-1, 3), vbar_s.reshape(-1, 3)])
        tbar, zbar, gbars = d.vjp(targets, lats, lam)
        mpbar_c, mpbar_s = tbar[:nc_].reshape(mp_c.shape), tbar[nc_:].reshape(mp_s.shape)
        Zb[:-1] += 0.5 * mpbar_c
        Zb[1:] += 0.5 * mpbar_c
        Zb[:, :-1] += 0.5 * mpbar_s
        Zb[:, 1:] += 0.5 * mpbar_s
        Zw += zbar[0]
        Zb += zbar[1]
        Gw += gbars[0]
        Gb += gbars[1]
        # unsteady force rho * gamma_dot * nc
        Gbd += rho * np.einsum("ijk,k->ij", nc, Fbar)
        ncbar = rho * gbd[..., None] * Fbar
        # 2. gamma_dot filter
        Gb += (relax / dt) * Gbd
        Gb_prev = -(relax / dt) * Gbd
        Gbd_prev = (1.0 - relax) * Gbd
        # 3. transpose solve with A_n
        factors = getattr(seg, "factors", None)
        mu = d.solve_t(zb, None, Gb) if factors is None else d.solve_t_factors(factors[0][loc], factors[1][loc], Gb)
        # 4. RHS + AIC geometry: b = -(U - c_dot + V_w(c)) . nc and A Gamma = nc . V_b(c)
        cdot = 0.5 * (0.5 * (zbd[:-1, :-1] + zbd[1:, :-1]) + 0.5 * (zbd[:-1, 1:] + zbd[1:, 1:]))
        Vtot = d.vind(c, [(zw, gw), (zb, gb)])
        ncbar += -mu[..., None] * (U - cdot + Vtot)
        cdotbar = mu[..., None] * nc
        lam_c = -mu[..., None] * nc
        cbar, zbar2, gbar2 = d.vjp(c, [(zw, gw), (zb, gb)], lam_c)
        Zw += zbar2[0]
        Zb += zbar2[1]
        Gw += gbar2[0]   # the bound part belongs to the solve's linearity in Gamma
        # 5. geometry
        Zb += _avg4_T(cbar, zb.shape)
        Zb += _normals_T(zb, ncbar)
        Zbd += _avg4_T(cdotbar, zbd.shape)
        # 6. wake shedding transposes; the free wake's convection velocity
        #    V(zw_{n-1}; bound n-1, wake n-1) adds its own VJP
        zw_nm1, gw_nm1 = seg.zeta_w[0][loc - 1], seg.gamma_w[0][loc - 1]
        zb_nm1, gb_nm1 = seg.zeta_b[0][loc - 1], seg.gamma_b[0][loc - 1]
        free = bool(self.uv.free_wake) and W > 0
        lats_nm1 = [(zb_nm1, gb_nm1), (zw_nm1, gw_nm1)]
        dw = self.uv.delta_w[0] if getattr(self.uv, "delta_w", None) else None
        if dw is not None:
            v_conv = d.vind(zw_nm1, lats_nm1) if free else None
            zw_p, te_bar, gte_bar, gw_p = _variable_wake_T(
                zw_nm1, zb[-1], gb_nm1[-1], gw_nm1, np.asarray(dw, float), dt, U, Zw, Gw, v_conv)
            Zb[-1] += te_bar
            Zw_prev = zw_p
            Gw_prev = gw_p
            Gb_prev[-1, :] += gte_bar
            conv_rows, conv_bar = slice(None), zw_p  # every row of zw_{n-1} is convected
        else:
            Zb[-1] += Zw[0]
            Zw_prev = np.zeros_like(Zw)
            Zw_prev[:-1] += Zw[1:]
            Gw_prev = np.zeros_like(Gw)
            if W > 0:
                Gb_prev[-1, :] += Gw[0, :]
                Gw_prev[:-1] += Gw[1:]
            conv_rows, conv_bar = slice(0, W), Zw[1:]
        Zb_prev = np.zeros_like(zb)
        if free:
            conv_bar = np.array(conv_bar)  # x_r = zw_{n-1,r} + dt (U + V(zw_{n-1,r})): lam = dt x_bar
            tbar, zbar_c, gbar_c = d.vjp(zw_nm1[conv_rows], lats_nm1, dt * conv_bar)
            Zw_prev[conv_rows] += tbar
            Zb_prev += zbar_c[0]
            Zw_prev += zbar_c[1]
            Gb_prev += gbar_c[0]
            Gw_prev += gbar_c[1]
        # 7. node frames
        zeta0_bar += _frames_T(Zb, Zbd, hg_n, hgd_n, dof)
        return Gb_prev, Gbd_prev, Gw_prev, Zw_prev, Zb_prev

    def _reverse_static(self, st, Gb0, Gw0, Zw0, Zb0, zeta0_bar, hg0, dof, m, n_, W, U):
        d = self.d
        zb = st.zeta_b[0]
        zw = st.zeta_w[0]
        gb = st.gamma_b[0]
        gw = st.gamma_w[0]
        nc = st.nc[0]
        c = st.c[0]
        Gb = Gb0.copy()
        Zw = Zw0.copy()
        if W > 0:
            Gb[-1, :] += Gw0.sum(axis=0)  # gamma_w = broadcast of the TE row (uvlm.py:995-1012)
        mu = d.solve_t(zb, zw if W > 0 else None, Gb)
        lats = [(zw, gw), (zb, gb)]
        Vtot = d.vind(c, lats)
        ncbar = -mu[..., None] * (U + Vtot)
        cbar, zbar, _ = d.vjp(c, lats, -mu[..., None] * nc)
        Zw += zbar[0]
        Zb = zbar[1] + Zb0
        Zb[-1] += Zw.sum(axis=0)  # every wake row = TE + s_r u_dir (uvlm.py:662-689)
        Zb += _avg4_T(cbar, zb.shape)
        Zb += _normals_T(zb, ncbar)
        zeta0_bar += _frames_T(Zb, None, hg0, None, dof)


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
