"""The aerodynamic time-step residual and its VJP (aero/uvlm.py:1942-2047, the function the
reference differentiates with jax.vjp inside the coupled adjoint's GMRES,
coupled/gradients/coupled.py:1215-1249).

``AeroResidual(uvlm).vjp(...)`` returns the residual and the cotangents of every input
for a cotangent r_bar of the residual, with the Biot-Savart sums and their VJPs, the AIC
and its factorisation on the device (fj_vind, fj_vind_vjp, fj_aic_assemble,
fj_lu_factor/solve/solve_t).  The inputs are the node frames of steps n and n-1 and the
frame velocities of step n; the reference reaches them from the beam coordinates through
beam code (``calculate_hg_from_varphi``, ``make_hg_dot``), which stays the caller's:
the hg cotangents returned here are what that chain rule consumes.

Residual blocks, in the reference's order (gamma_b, gamma_w, gamma_dot, zeta_w, f):

* r_gamma_b = solve(A_n, -(u - c_dot + V_w(c)) . n) - gamma_b_n  (:1529-1645);
* r_gamma_w, r_zeta_w = propagate_wake(q_{n-1}, zeta_b_n) - (gamma_w_n, zeta_w_n) (:1647-1751);
* r_gamma_dot = g/dt (gamma_b_n - gamma_b_{n-1}) + (1-g) gamma_dot_{n-1} - gamma_dot_n (:1753-1801);
* r_f = R^T P(f_steady + f_unsteady) - f_beam_n, P the projection onto the beam nodes
  (aero/utils.py:666-697) and R the node rotations (:1803-1940).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .adjoint import _avg4_T, _Dev, _flow_T, _normals_T, _variable_wake_T

_STATES = ("gamma_b", "gamma_w", "gamma_b_dot", "zeta_w")


def _frames(hg, zeta0, dof):
    """zeta = R zeta0 + t per vertex column (uvlm.py:537-561; hg_dot the same with Rdot)."""
    h = hg[dof]
    return np.einsum("jkl,ijl->ijk", h[:, :3, :3], zeta0) + h[None, :, :3, 3]


def _frames_hg_T(zbar, zeta0, dof, n_nodes):
    """hg cotangent (n_nodes, 4, 4) of zeta = R zeta0 + t."""
    out = np.zeros((n_nodes, 4, 4))
    np.add.at(out, (dof, slice(0, 3), slice(0, 3)), np.einsum("ijk,ijl->jkl", zbar, zeta0))
    np.add.at(out, (dof, slice(0, 3), 3), zbar.sum(axis=0))
    return out


class AeroResidual:
    """Residual and VJP for one UVLM (FP64, epsilon or cutoff kernel, any number of
    surfaces, prescribed or free wake, uniform or delta_w, Constant or gust flow)."""

    def __init__(self, uvlm, device=None, dev=None):
        self.uv = uvlm
        if dev is None:
            if uvlm.kernel.kernel_id not in (_lib.FJ_KERNEL_EPSILON, _lib.FJ_KERNEL_CUTOFF):
                raise NotImplementedError("the residual VJP is written for the epsilon and cutoff kernels")
            mirror = None if uvlm.mirror_point is None else (uvlm.mirror_point, uvlm.mirror_normal)
            dev = _Dev(device, uvlm.kernel.kernel_id, uvlm.kernel.r_cut, mirror)
        self.d = dev
        self.include_unsteady = bool(getattr(uvlm, "include_unsteady_force", True))

    # -- helpers -------------------------------------------------------------------
    def _lattices(self, hg_n, hg_dot_n, hg_nm1):
        uv = self.uv
        z0 = [np.asarray(z, float) for z in uv.zeta_b0]
        dof = [np.asarray(d) for d in uv.dof_mapping]
        zb = [_frames(hg_n, z, d) for z, d in zip(z0, dof)]
        zbd = [np.einsum("jkl,ijl->ijk", hg_dot_n[d][:, :3, :3], z) + hg_dot_n[d][None, :, :3, 3]
               for z, d in zip(z0, dof)]
        zb1 = [_frames(hg_nm1, z, d) for z, d in zip(z0, dof)]
        return z0, dof, zb, zbd, zb1

    @staticmethod
    def ravel(q):
        """AeroStates order (aero/gradients/data_structures.py:165-178)."""
        return np.concatenate([np.concatenate([np.ravel(a) for a in q[k]]) for k in _STATES])

    # -- residual and VJP ----------------------------------------------------------------
    def vjp(self, t_n, hg_n, hg_dot_n, hg_nm1, q_n, q_nm1, f_beam_n, r_bar):
        """(residual, cotangents): r_bar is the cotangent of the residual (the reference's
        concatenation); the cotangents are a dict with q_n, q_nm1 (dicts of per-surface
        lists), hg_n, hg_dot_n, hg_nm1 and f_beam_n."""
        d, uv = self.d, self.uv
        ff = uv.flowfield
        rho, dt, g = ff.rho, uv.dt, uv.gamma_dot_relaxation
        hg_n, hg_dot_n, hg_nm1 = (np.asarray(a, float) for a in (hg_n, hg_dot_n, hg_nm1))
        n_nodes = hg_n.shape[0]
        S = uv.n_surf
        sl = range(S)
        z0, dof, zb, zbd, zb1 = self._lattices(hg_n, hg_dot_n, hg_nm1)
        gb, gw, gbd, zw = ([np.asarray(a, float) for a in q_n[k]] for k in _STATES)
        gb1, gw1, gbd1, zw1 = ([np.asarray(a, float) for a in q_nm1[k]] for k in _STATES)
        f_beam_n = np.asarray(f_beam_n, float).reshape(n_nodes, 6)
        # split r_bar into its blocks
        sizes = ([a.size for a in gb], [a.size for a in gw], [a.size for a in gbd], [a.size for a in zw])
        rb, off = [], 0
        for blk, shapes in zip(sizes, (gb, gw, gbd, zw)):
            parts = []
            for k, a in zip(blk, shapes):
                parts.append(np.asarray(r_bar[off:off + k], float).reshape(a.shape))
                off += k
            rb.append(parts)
        rb_gb, rb_gw, rb_gbd, rb_zw = rb
        rb_f = np.asarray(r_bar[off:off + n_nodes * 6], float).reshape(n_nodes, 6)
        # cotangent accumulators
        Gb = [np.zeros_like(a) for a in gb]
        Gw = [np.zeros_like(a) for a in gw]
        Gbd = [np.zeros_like(a) for a in gbd]
        Zw = [np.zeros_like(a) for a in zw]
        Gb1 = [np.zeros_like(a) for a in gb1]
        Gw1 = [np.zeros_like(a) for a in gw1]
        Gbd1 = [np.zeros_like(a) for a in gbd1]
        Zw1 = [np.zeros_like(a) for a in zw1]
        Zb = [np.zeros_like(a) for a in zb]
        Zbd = [np.zeros_like(a) for a in zbd]
        Zb1 = [np.zeros_like(a) for a in zb1]
        res = []

        # -- 1. bound circulation: x = solve(A, -b), r = x - gamma_b -----------------------
        c = [0.5 * (0.5 * (z[:-1, :-1] + z[1:, :-1]) + 0.5 * (z[:-1, 1:] + z[1:, 1:])) for z in zb]
        nc = [np.cross(z[1:, 1:] - z[:-1, :-1], z[1:, :-1] - z[:-1, 1:]) for z in zb]
        cdot = [0.5 * (0.5 * (z[:-1, :-1] + z[1:, :-1]) + 0.5 * (z[:-1, 1:] + z[1:, 1:])) for z in zbd]
        co = np.concatenate([[0], np.cumsum([x.shape[0] * x.shape[1] for x in c])])
        c_all = np.concatenate([x.reshape(-1, 3) for x in c])
        wakes = [(zw[s], gw[s]) for s in sl]
        v_w = d.vind(c_all, wakes) if any(a.size for a in gw) else np.zeros_like(c_all)
        b = np.concatenate([np.einsum("ijk,ijk->ij",
                                      ff(c[s], t_n) - cdot[s] + v_w[co[s]:co[s + 1]].reshape(c[s].shape),
                                      nc[s]).ravel() for s in sl])
        rb_flat = np.concatenate([a.ravel() for a in rb_gb])
        x, mu_flat = d.solve_pair(zb, -b, rb_flat)
        po = np.concatenate([[0], np.cumsum([a.size for a in gb])])
        xs = [x[po[s]:po[s + 1]].reshape(gb[s].shape) for s in sl]
        mu = [mu_flat[po[s]:po[s + 1]].reshape(gb[s].shape) for s in sl]
        res.append(np.concatenate([(xs[s] - gb[s]).ravel() for s in sl]))
        for s in sl:
            Gb[s] -= rb_gb[s]
        lats_x = wakes + [(zb[s], xs[s]) for s in sl]
        v_x = d.vind(c_all, [(zb[s], xs[s]) for s in sl])
        lam_c = [-mu[s][..., None] * nc[s] for s in sl]
        ncbar = []
        for s in sl:
            v_all = v_w[co[s]:co[s + 1]] + v_x[co[s]:co[s + 1]]
            ncbar.append(-mu[s][..., None] * (ff(c[s], t_n) - cdot[s] + v_all.reshape(c[s].shape)))
        cbar_all, zbar, gbar = d.vjp(c_all, lats_x, np.concatenate([a.reshape(-1, 3) for a in lam_c]))
        for s in sl:
            cbar = cbar_all[co[s]:co[s + 1]].reshape(c[s].shape) + _flow_T(ff, c[s], t_n, lam_c[s])
            Zw[s] += zbar[s]
            Gw[s] += gbar[s]
            Zb[s] += zbar[S + s]   # gamma = x: the solve's own linearity
            Zb[s] += _avg4_T(cbar, zb[s].shape)
            Zbd[s] += _avg4_T(mu[s][..., None] * nc[s], zbd[s].shape)

        # -- 2. wake: (zeta_w, gamma_w) = propagate(q_{n-1}, zeta_b_n) ---------------------------
        lats_nm1 = [(zb1[s], gb1[s]) for s in sl] + [(zw1[s], gw1[s]) for s in sl]
        free = bool(uv.free_wake)
        dws = getattr(uv, "delta_w", None) or [None] * S
        conv = []
        r_zw, r_gw = [], []
        for s in sl:
            W = gw[s].shape[0]
            Zw[s] -= rb_zw[s]
            Gw[s] -= rb_gw[s]
            ucv = ff(zw1[s], t_n)
            if dws[s] is not None:
                v_conv = d.vind(zw1[s], lats_nm1) if (free and W > 0) else None
                vel = ucv if v_conv is None else ucv + v_conv
                znew, gnew = _propagate_var(zw1[s], zb[s][-1], gb1[s][-1], gw1[s], np.asarray(dws[s], float), dt, vel)
                zw_p, te_bar, gte_bar, gw_p = _variable_wake_T(zw1[s], zb[s][-1], gb1[s][-1], gw1[s],
                                                               np.asarray(dws[s], float), dt, ucv, rb_zw[s], rb_gw[s],
                                                               v_conv)
                Zb[s][-1] += te_bar
                Zw1[s] += zw_p
                Gw1[s] += gw_p
                Gb1[s][-1, :] += gte_bar
                rows, cb = slice(None), np.array(zw_p)
            else:
                v_rows = ucv[:-1]
                if free and W > 0:
                    v_rows = v_rows + d.vind(zw1[s][:-1], lats_nm1)
                znew = np.concatenate([zb[s][-1][None], zw1[s][:-1] + dt * v_rows], axis=0)
                gnew = np.concatenate([gb1[s][-1][None], gw1[s][:-1]], axis=0) if W > 0 else np.zeros_like(gw1[s])
                Zb[s][-1] += rb_zw[s][0]
                Zw1[s][:-1] += rb_zw[s][1:]
                if W > 0:
                    Gb1[s][-1, :] += rb_gw[s][0, :]
                    Gw1[s][:-1] += rb_gw[s][1:]
                rows, cb = slice(0, W), np.array(rb_zw[s][1:])
            r_zw.append(znew - zw[s])
            r_gw.append(gnew - gw[s])
            Zw1[s][rows] += dt * _flow_T(ff, zw1[s][rows], t_n, cb)
            conv.append((rows, cb))
        if free:
            tparts = [zw1[s][conv[s][0]].reshape(-1, 3) for s in sl]
            to = np.concatenate([[0], np.cumsum([p.shape[0] for p in tparts])])
            if to[-1] > 0:
                lam = np.concatenate([dt * conv[s][1].reshape(-1, 3) for s in sl])
                tbar, zbar_c, gbar_c = d.vjp(np.concatenate(tparts), lats_nm1, lam)
                for s in sl:
                    Zw1[s][conv[s][0]] += tbar[to[s]:to[s + 1]].reshape(zw1[s][conv[s][0]].shape)
                    Zb1[s] += zbar_c[s]
                    Zw1[s] += zbar_c[S + s]
                    Gb1[s] += gbar_c[s]
                    Gw1[s] += gbar_c[S + s]
        res.append(np.concatenate([a.ravel() for a in r_gw]))

        # -- 3. gamma_dot ------------------------------------------------------------------
        res.append(np.concatenate([(g / dt * (gb[s] - gb1[s]) + (1.0 - g) * gbd1[s] - gbd[s]).ravel() for s in sl]))
        for s in sl:
            Gb[s] += g / dt * rb_gbd[s]
            Gb1[s] -= g / dt * rb_gbd[s]
            Gbd1[s] += (1.0 - g) * rb_gbd[s]
            Gbd[s] -= rb_gbd[s]
        res.append(np.concatenate([a.ravel() for a in r_zw]))

        # -- 4. forces: r = R^T P(F) - f_beam ----------------------------------------------------
        lats = [(zb[s], gb[s]) for s in sl] + [(zw[s], gw[s]) for s in sl]
        mp_c = [0.5 * (z[:-1] + z[1:]) for z in zb]
        mp_s = [0.5 * (z[:, :-1] + z[:, 1:]) for z in zb]
        parts = []
        for s in sl:
            parts += [mp_c[s].reshape(-1, 3), mp_s[s].reshape(-1, 3)]
        offs = np.concatenate([[0], np.cumsum([p.shape[0] for p in parts])])
        targets = np.concatenate(parts)
        v = d.vind(targets, lats)
        F, geo = [], []
        for s in sl:
            m, n_ = gb[s].shape
            v_c = v[offs[2 * s]:offs[2 * s + 1]].reshape(mp_c[s].shape)
            v_s = v[offs[2 * s + 1]:offs[2 * s + 2]].reshape(mp_s[s].shape)
            vr_c = ff(mp_c[s], t_n) + v_c - 0.5 * (zbd[s][:-1] + zbd[s][1:])
            vr_s = ff(mp_s[s], t_n) + v_s - 0.5 * (zbd[s][:, :-1] + zbd[s][:, 1:])
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
            f_c = rho * g_c[..., None] * np.cross(vr_c, r_c)
            f_s = rho * g_s[..., None] * np.cross(vr_s, r_s)
            fv = np.zeros_like(zb[s])
            fv[:-1] += 0.5 * f_c
            fv[1:] += 0.5 * f_c
            fv[:, :-1] += 0.5 * f_s
            fv[:, 1:] += 0.5 * f_s
            if self.include_unsteady:
                fu = rho * gbd[s][..., None] * nc[s]
                fv[:-1, :-1] += 0.25 * fu
                fv[1:, :-1] += 0.25 * fu
                fv[:-1, 1:] += 0.25 * fu
                fv[1:, 1:] += 0.25 * fu
            F.append(fv)
            geo.append((vr_c, vr_s, g_c, g_s, r_c, r_s))
        Rm = hg_n[:, :3, :3]
        G = np.zeros((n_nodes, 6))
        arms = []
        for s in sl:
            arm = np.einsum("jkl,ijl->ijk", Rm[dof[s]], z0[s])  # R_j x0[i, j]
            arms.append(arm)
            G[dof[s], :3] = F[s].sum(axis=0)
            G[dof[s], 3:] = np.cross(arm, F[s]).sum(axis=0)
        L_lin = np.einsum("jkl,jk->jl", Rm, G[:, :3])   # R^T G
        L_rot = np.einsum("jkl,jk->jl", Rm, G[:, 3:])
        res.append((np.concatenate([L_lin, L_rot], axis=1) - f_beam_n).ravel())
        f_beam_bar = -rb_f
        # R^T G: G_bar = R L_bar, R_bar += G L_bar^T
        Gbar = np.concatenate([np.einsum("jkl,jl->jk", Rm, rb_f[:, :3]), np.einsum("jkl,jl->jk", Rm, rb_f[:, 3:])], 1)
        Rbar = np.einsum("jk,jl->jkl", G[:, :3], rb_f[:, :3]) + np.einsum("jk,jl->jkl", G[:, 3:], rb_f[:, 3:])
        lam = np.zeros_like(targets)
        fbars = []
        written = np.zeros(n_nodes, bool)
        for s in reversed(sl):  # the last surface to write a node owns it
            own = ~written[dof[s]]
            written[dof[s]] = True
            gl = np.where(own[:, None], Gbar[dof[s], :3], 0.0)
            gr = np.where(own[:, None], Gbar[dof[s], 3:], 0.0)
            Fb = np.broadcast_to(gl[None], F[s].shape) + np.cross(gr[None], arms[s])
            arm_bar = np.cross(F[s], np.broadcast_to(gr[None], F[s].shape))
            np.add.at(Rbar, dof[s], np.einsum("ijk,ijl->jkl", arm_bar, z0[s]))
            fbars.append((s, Fb))
        for s, Fb in fbars:
            vr_c, vr_s, g_c, g_s, r_c, r_s = geo[s]
            fc_bar = 0.5 * (Fb[:-1] + Fb[1:])
            fs_bar = 0.5 * (Fb[:, :-1] + Fb[:, 1:])
            gbar_c = rho * np.einsum("ijk,ijk->ij", np.cross(vr_c, r_c), fc_bar)
            gbar_s = rho * np.einsum("ijk,ijk->ij", np.cross(vr_s, r_s), fs_bar)
            vbar_c = rho * g_c[..., None] * np.cross(r_c, fc_bar)
            vbar_s = rho * g_s[..., None] * np.cross(r_s, fs_bar)
            rbar_c = rho * g_c[..., None] * np.cross(fc_bar, vr_c)
            rbar_s = rho * g_s[..., None] * np.cross(fs_bar, vr_s)
            Zb[s][1:] += rbar_c
            Zb[s][:-1] -= rbar_c
            Zb[s][:, 1:] += rbar_s
            Zb[s][:, :-1] -= rbar_s
            Zbd[s][:-1] += -0.5 * vbar_c
            Zbd[s][1:] += -0.5 * vbar_c
            Zbd[s][:, :-1] += -0.5 * vbar_s
            Zbd[s][:, 1:] += -0.5 * vbar_s
            Gb[s] += gbar_c[:, :-1] - gbar_c[:, 1:] - gbar_s[:-1, :] + gbar_s[1:, :]
            if gw[s].shape[0] > 0:
                Gw[s][0, :] -= gbar_s[-1, :]
            lam[offs[2 * s]:offs[2 * s + 1]] = vbar_c.reshape(-1, 3)
            lam[offs[2 * s + 1]:offs[2 * s + 2]] = vbar_s.reshape(-1, 3)
            mpbar_c = _flow_T(ff, mp_c[s], t_n, vbar_c)
            mpbar_s = _flow_T(ff, mp_s[s], t_n, vbar_s)
            Zb[s][:-1] += 0.5 * mpbar_c
            Zb[s][1:] += 0.5 * mpbar_c
            Zb[s][:, :-1] += 0.5 * mpbar_s
            Zb[s][:, 1:] += 0.5 * mpbar_s
            if self.include_unsteady:
                ub = 0.25 * (Fb[:-1, :-1] + Fb[1:, :-1] + Fb[:-1, 1:] + Fb[1:, 1:])
                Gbd[s] += rho * np.einsum("ijk,ijk->ij", nc[s], ub)
                ncbar[s] += rho * gbd[s][..., None] * ub
        tbar, zbar, gbar = d.vjp(targets, lats, lam)
        for s in sl:
            mpbar_c = tbar[offs[2 * s]:offs[2 * s + 1]].reshape(mp_c[s].shape)
            mpbar_s = tbar[offs[2 * s + 1]:offs[2 * s + 2]].reshape(mp_s[s].shape)
            Zb[s][:-1] += 0.5 * mpbar_c
            Zb[s][1:] += 0.5 * mpbar_c
            Zb[s][:, :-1] += 0.5 * mpbar_s
            Zb[s][:, 1:] += 0.5 * mpbar_s
            Zb[s] += zbar[s]
            Gb[s] += gbar[s]
            Zw[s] += zbar[S + s]
            Gw[s] += gbar[S + s]
            Zb[s] += _normals_T(zb[s], ncbar[s])

        # -- node frames ------------------------------------------------------------------
        hg_bar = np.zeros_like(hg_n)
        hgd_bar = np.zeros_like(hg_dot_n)
        hg1_bar = np.zeros_like(hg_nm1)
        for s in sl:
            hg_bar += _frames_hg_T(Zb[s], z0[s], dof[s], n_nodes)
            hgd_bar += _frames_hg_T(Zbd[s], z0[s], dof[s], n_nodes)
            hg1_bar += _frames_hg_T(Zb1[s], z0[s], dof[s], n_nodes)
        hg_bar[:, :3, :3] += Rbar
        cot = {"q_n": dict(zip(_STATES, (Gb, Gw, Gbd, Zw))), "q_nm1": dict(zip(_STATES, (Gb1, Gw1, Gbd1, Zw1))),
               "hg_n": hg_bar, "hg_dot_n": hgd_bar, "hg_nm1": hg1_bar, "f_beam_n": f_beam_bar}
        return np.concatenate(res), cot


def _propagate_var(zw1, te, gte, gw1, dw, dt, vel):
    """propagate_surf_wake with delta_w (aero/utils.py:452-491) for one surface: the
    convected rows re-interpolated onto the prescribed arc lengths."""
    X = np.concatenate([te[None], zw1 + dt * vel], axis=0)
    G = np.concatenate([gte[None], gw1], axis=0)
    seg = np.linalg.norm(X[1:] - X[:-1], axis=-1)
    S = np.concatenate([np.zeros((1, X.shape[1])), np.cumsum(seg, axis=0)], axis=0)
    SG = 0.5 * (0.5 * (S[:-1, :-1] + S[1:, :-1]) + 0.5 * (S[:-1, 1:] + S[1:, 1:]))
    s_disc = np.concatenate([np.zeros(1), np.cumsum(dw)])
    sg_disc = 0.5 * (s_disc[:-1] + s_disc[1:])
    zn = np.stack([np.stack([np.interp(s_disc, S[:, j], X[:, j, k]) for k in range(3)], -1)
                   for j in range(X.shape[1])], 1)
    gn = np.stack([np.interp(sg_disc, SG[:, j], G[:, j]) for j in range(G.shape[1])], 1) if gw1.size else gw1.copy()
    return zn, gn
