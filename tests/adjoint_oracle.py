"""The reverse sweep of ``flapjax_b200.adjoint.PrescribedAdjoint`` with the oracle standing
in for the device: forward runs, induced velocities, Biot-Savart VJPs and the transposed
AIC solve come from the FP64 NumPy restatement.  Lets the CPU suite check the sweep's
algebra (every transpose, the checkpointing) against finite differences of the oracle
forward; the GPU tests check the same sweep on the device kernels."""
from __future__ import annotations

import numpy as np

from flapjax_b200 import cases
from flapjax_b200.adjoint import PrescribedAdjoint
from oracle import uvlm_ref as R
from oracle.uvlm_vjp import bs_vjp

_KEYS = ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady", "f_unsteady",
         "alpha")


class _Snap:
    """One slot of an oracle Case, shaped like a snapshot AeroCase."""

    def __init__(self, case, i):
        for k in _KEYS:
            setattr(self, k, [a[i] for a in getattr(case, k)])
        self.t = case.t[i]
        self._case, self._i = case, i


class _Seg:
    def __init__(self, case):
        for k in _KEYS:
            setattr(self, k, getattr(case, k))
        self.force_total = sum(fs.sum(axis=(1, 2)) + fu.sum(axis=(1, 2))
                               for fs, fu in zip(case.f_steady, case.f_unsteady))
        self.t = case.t
        self._case = case

    def __getitem__(self, i):
        return _Snap(self._case, i)


class OracleDev:
    def __init__(self, kernel=R.KERNEL_EPSILON, r_cut=R.R_CUTOFF, mirror=None):
        self.kernel = kernel
        self.r_cut = r_cut
        self.mirror = mirror

    def vind(self, targets, lats):
        return R.compute_v_ind(targets, [z for z, _ in lats], [g for _, g in lats], self.kernel, self.mirror,
                               self.r_cut)

    def vjp(self, targets, lats, lam):
        """With a mirror plane the image lattice (reflected vertices, strengths negated)
        adds its VJP, reflected back onto the original vertices."""
        tb, zb, gb = self._vjp(targets, lats, lam)
        if self.mirror is None:
            return tb, zb, gb
        p, nrm = (np.asarray(v, float) for v in self.mirror)
        refl = np.eye(3) - 2.0 * np.outer(nrm, nrm)
        tb2, zb2, gb2 = self._vjp(targets, [(R.mirror_grid(z, p, nrm), -g) for z, g in lats], lam)
        return (tb + tb2, [a + b @ refl.T for a, b in zip(zb, zb2)], [a - b for a, b in zip(gb, gb2)])

    def _vjp(self, targets, lats, lam):
        t = targets.reshape(-1, 3)
        lm = lam.reshape(-1, 3)
        tb = np.zeros_like(t)
        zb, gb = [], []
        for z, g in lats:
            g_m, g_n = R.gamma_eff(g)
            zbar = np.zeros_like(z)
            gbar_m = np.zeros_like(g_m)
            gbar_n = np.zeros_like(g_n)
            for segs, gs, gbar, kind in ((R.chordwise_segments(z), g_m, gbar_m, "m"),
                                          (R.spanwise_segments(z), g_n, gbar_n, "n")):
                y0, y1 = segs[..., 0, :], segs[..., 1, :]
                kv = R.kernel_eval(self.kernel, t[:, None, None, :], y0[None], y1[None], self.r_cut)
                gbar += np.einsum("tijk,tk->ij", kv, lm)
                xb, y0b, y1b = bs_vjp(t[:, None, None, :], y0[None], y1[None],
                                      lm[:, None, None, :] * gs[None, ..., None], self.kernel, self.r_cut)
                tb += xb.sum(axis=(1, 2))
                y0b, y1b = y0b.sum(0), y1b.sum(0)
                if kind == "m":      # chordwise filament (k,l): zeta[k,l] -> zeta[k+1,l]
                    zbar[:-1] += y0b
                    zbar[1:] += y1b
                else:                # spanwise filament (k,l): zeta[k,l] -> zeta[k,l+1]
                    zbar[:, :-1] += y0b
                    zbar[:, 1:] += y1b
            # g_m = diff(pad(G, cols), axis=1), g_n = -diff(pad(G, rows), axis=0)
            Gb = gbar_m[:, :-1] - gbar_m[:, 1:] - gbar_n[:-1, :] + gbar_n[1:, :]
            zb.append(zbar)
            gb.append(Gb)
        return tb.reshape(targets.shape), zb, gb

    def solve_pair(self, zetas_b, rhs, rhs_t):
        cs = [R.compute_surf_c(z) for z in zetas_b]
        ns = [R.compute_surf_nc(z) for z in zetas_b]
        a = R.compute_aic_solve(cs, ns, list(zetas_b), None, self.kernel, self.mirror, self.r_cut)
        return R._solve(a, np.ravel(rhs)), np.linalg.solve(a.T, np.ravel(rhs_t))

    def solve_t(self, zetas_b, zetas_w_static, rhs):
        cs = [R.compute_surf_c(z) for z in zetas_b]
        ns = [R.compute_surf_nc(z) for z in zetas_b]
        a = R.compute_aic_solve(cs, ns, list(zetas_b), None if zetas_w_static is None else list(zetas_w_static),
                                self.kernel, self.mirror, self.r_cut)
        return np.linalg.solve(a.T, np.ravel(rhs)).reshape(np.shape(rhs))


class OracleAdjoint(PrescribedAdjoint):
    """``PrescribedAdjoint`` over an oracle ``UVLMRef`` (same attribute names)."""

    def __init__(self, ref):
        self.uv = ref
        self.d = OracleDev(ref.kernel, ref.r_cut, ref.mirror)

    def _static(self):
        return _Snap(self.uv.solve_static(), 0)

    def _run_segment(self, init, hg_seg, hgd_seg, keep_factors=False):
        return _Seg(self.uv.solve_prescribed_dynamic(init._case if init._i == 0 else _one(init), hg_seg, hgd_seg))


def _one(snap):
    """An oracle Case holding only ``snap`` (slot 0)."""
    case = snap._case
    out = R.Case(**{k: [a[snap._i:snap._i + 1] for a in getattr(case, k)] for k in _KEYS}, t=case.t[snap._i:snap._i + 1])
    return out


def forward_objective(case, zeta_b0, fw, delta_w=None):
    """J = sum_{n>=1} fw[n] . F_n of the oracle forward at the lattice ``zeta_b0`` (in
    the oracle's current floating type), with an optional variable wake ``delta_w``."""
    from flapjax_b200 import cases
    from tests.helpers import oracle_uvlm

    uv, ff = oracle_uvlm(cases.WingCase(**{**case.__dict__, "zeta_b0": zeta_b0}))
    if delta_w is not None:
        uv.set_design_variables(case.dt, ff, zeta_b0, case.hg0, delta_w=np.asarray(delta_w, float))
    out = uv.solve_prescribed_dynamic(uv.solve_static(), case.hg_t, case.hg_dot_t)
    ft = sum(fs.sum(axis=(1, 2)) + fu.sum(axis=(1, 2)) for fs, fu in zip(out.f_steady, out.f_unsteady))
    return np.sum(fw[1:] * ft[1:])


def central_difference(case, direction, fw, h=1e-6, delta_w=None):
    """(J(z + h d) - J(z - h d)) / 2h of the oracle forward run in 80-bit extended
    precision.  In float64 the forward carries ~1e-11 relative roundoff noise (the
    epsilon kernel evaluated at a filament's own midpoint divides roundoff by
    eps |r0|^2), which limits a float64 central difference at h = 1e-6 to ~1e-4."""
    z = np.asarray(case.zeta_b0, np.longdouble)
    hh = np.longdouble(h)
    with R.real_type(np.longdouble):
        jp = forward_objective(case, z + hh * direction, fw, delta_w)
        jm = forward_objective(case, z - hh * direction, fw, delta_w)
    return float((jp - jm) / (2 * hh))


def coefficient_weights(case, which):
    """fw with fw[n] . F_n / ... = time average over steps 1..N of CL or CD."""
    a = np.deg2rad(case.alpha_deg)
    e = np.array((-np.sin(a), 0.0, np.cos(a))) if which == "CL" else np.array((np.cos(a), 0.0, np.sin(a)))
    q = 0.5 * case.rho * case.u_mag**2 * case.s_ref
    fw = np.zeros((case.n_tstep, 3))
    fw[1:] = e / (q * case.n_steps)
    return fw


def two_surface_case(free_wake=False, n_steps=3):
    """A 3 x 4 heaving wing and a 2 x 2 tail 3 chords behind it on their own nodes (the
    layout of the two-surface golden case), as (surfaces, hg0, hg_t, hg_dot_t, wing)."""
    wing = (cases.wing_free(m=3, n=4, m_star=4, n_steps=n_steps, seed=1) if free_wake
            else cases.wing_heave(m=3, n=4, m_star=4, n_steps=n_steps))
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
    surfs = [(3, 4, 4, np.asarray(wing.zeta_b0, float), np.arange(5)), (2, 2, 3, tail, np.arange(5, 8))]
    return surfs, hg0, hg_t, hg_dot_t, wing


def two_surface_oracle(surfs, hg0, wing, zetas=None):
    uv = R.UVLMRef([(m, n, ms) for m, n, ms, _, _ in surfs], [d for *_, d in surfs], kernel=wing.kernel,
                   r_cut=wing.r_cut, free_wake=wing.free_wake)
    uv.set_design_variables(wing.dt, R.Constant(wing.u_inf, wing.rho, True),
                            [z for *_, z, _ in surfs] if zetas is None else zetas, hg0)
    return uv
