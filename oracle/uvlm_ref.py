"""FP64 CPU oracle for the FLAPJAX UVLM hot path (TEST INFRASTRUCTURE ONLY).

This module restates, in NumPy float64, the arithmetic of the reference's unsteady
vortex-lattice path so that the CUDA library can be checked against it.  It is the
checker, never the product: only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.

Parity status: the reference (ben-l-p/flapjax 1.2.1) is pure JAX and JAX is not
installed on these machines, so the reference cannot run natively.  This oracle is
pinned (a) by the reference's own known-answer and property tests
(``tests/algebra/test_kernels.py``, ``tests/aero/test_static_no_wake.py``,
``tests/aero/test_mirrored_wing.py``, ``tests/aero/test_variable_wake_disc.py``), and
(b) by golden vectors produced by executing the reference's own Python source under a
NumPy stand-in for ``jax`` (``tests/golden/make_golden.py``).  (b) runs the reference's
control flow and formulas, with NumPy's float64 arithmetic in place of XLA's.

Every function cites the reference file:line it follows (paths relative to
``src/flapjax/``).  Array layouts are the reference's: a lattice ``zeta`` is
``(rows+1, cols+1, 3)`` C-contiguous float64 and circulations are ``(rows, cols)``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.linalg

# utils/constants.py:13,16,19
HORSESHOE_LENGTH = 1e3
EPSILON = 1e-7
R_CUTOFF = 1e-4

KERNEL_EPSILON = "epsilon"
KERNEL_CUTOFF = "cutoff"
KERNEL_PLAIN = "plain"

_PAIR_BUDGET = 1 << 21  # (target, segment) pairs evaluated per NumPy chunk

# Floating type of every array the oracle creates.  float64 (the reference's type)
# unless a test switches to np.longdouble through ``real_type`` to take finite
# differences of the forward below the float64 roundoff floor.
REAL = np.float64


class real_type:
    """Context manager: run the oracle in another floating type (np.longdouble)."""

    def __init__(self, dtype):
        self.dtype = dtype

    def __enter__(self):
        global REAL
        self._old, REAL = REAL, self.dtype
        return self

    def __exit__(self, *exc):
        global REAL
        REAL = self._old


def _solve(a, b):
    """Dense solve: LAPACK getrf/getrs in float64; Gaussian elimination with partial
    pivoting (row by row, in the array's own type) for extended precision."""
    if a.dtype == np.float64 and b.dtype == np.float64:
        return scipy.linalg.lu_solve(scipy.linalg.lu_factor(a), b)
    a = a.astype(REAL).copy()
    x = b.astype(REAL).copy()
    n = a.shape[0]
    for k in range(n):
        p = k + int(np.argmax(np.abs(a[k:, k])))
        if p != k:
            a[[k, p]] = a[[p, k]]
            x[[k, p]] = x[[p, k]]
        f = a[k + 1:, k] / a[k, k]
        a[k + 1:, k:] -= f[:, None] * a[k, k:]
        x[k + 1:] -= f * x[k]
    for k in range(n - 1, -1, -1):
        x[k] = (x[k] - a[k, k + 1:] @ x[k + 1:]) / a[k, k]
    return x


# ----------------------------------------------------------------------------------
# Biot-Savart segment kernels, aero/utils.py:580-648.  Vectorised: x (..., 3),
# y0/y1 (..., 3) broadcast against each other; result (..., 3).
# ----------------------------------------------------------------------------------
def _dot(a, b):
    return np.sum(a * b, axis=-1)


def bs_plain(x, y0, y1):
    """``biot_savart`` aero/utils.py:580-592 (unregularised; NaN on the filament line)."""
    r0 = y1 - y0
    r1 = x - y0
    r2 = x - y1
    r1_x_r2 = np.cross(r1, r2)
    with np.errstate(divide="ignore", invalid="ignore"):
        diff_r = r1 / np.linalg.norm(r1, axis=-1)[..., None] - r2 / np.linalg.norm(
            r2, axis=-1
        )[..., None]
        return (
            r1_x_r2
            / (_dot(r1_x_r2, r1_x_r2) * 4.0 * np.pi)[..., None]
            * _dot(r0, diff_r)[..., None]
        )


def bs_epsilon(x, y0, y1):
    """``biot_savart_epsilon`` aero/utils.py:606-623, the reference's default kernel."""
    r0 = y1 - y0
    r1 = x - y0
    r2 = x - y1
    inv_n1 = 1.0 / np.sqrt(_dot(r1, r1) + EPSILON * EPSILON)
    inv_n2 = 1.0 / np.sqrt(_dot(r2, r2) + EPSILON * EPSILON)
    diff_r = r1 * inv_n1[..., None] - r2 * inv_n2[..., None]
    r1_x_r2 = np.cross(r1, r2)
    r0_sq = _dot(r0, r0)
    denom = _dot(r1_x_r2, r1_x_r2) + EPSILON * r0_sq * r0_sq
    return r1_x_r2 * (_dot(r0, diff_r) / (4.0 * np.pi * denom))[..., None]


def _unit_epsilon(r):
    """``make_unit_epsilon`` aero/utils.py:595-603."""
    return r / np.sqrt(_dot(r, r) + EPSILON**2)[..., None]


def bs_cutoff(x, y0, y1, r_cut=R_CUTOFF):
    """``biot_savart_cutoff`` aero/utils.py:626-648 with a run-time cutoff radius.

    The reference hard-wires ``R_CUTOFF`` (utils/constants.py:19); the radius is a
    parameter here so that a vortex-core radius can be set per case.
    """
    r0 = y1 - y0
    r1 = x - y0
    r2 = x - y1
    with np.errstate(divide="ignore", invalid="ignore"):
        sm = _dot(r0, r1) / _dot(r0, y1 - y0)
        m = y0 + sm[..., None] * (y1 - y0)
        r = np.linalg.norm(x - m, axis=-1)
        r1_x_r2 = np.cross(r1, r2)
        r1_x_r2_unit2 = r1_x_r2 / _dot(r1_x_r2, r1_x_r2)[..., None]
        diff_r = _unit_epsilon(r1) - _unit_epsilon(r2)
        val = r1_x_r2_unit2 / (4.0 * np.pi) * _dot(r0, diff_r)[..., None]
    return np.where((r > r_cut)[..., None], val, 0.0)


def kernel_eval(kernel, x, y0, y1, r_cut=R_CUTOFF):
    if kernel == KERNEL_EPSILON:
        return bs_epsilon(x, y0, y1)
    if kernel == KERNEL_CUTOFF:
        return bs_cutoff(x, y0, y1, r_cut)
    if kernel == KERNEL_PLAIN:
        return bs_plain(x, y0, y1)
    raise ValueError(f"unknown kernel {kernel!r}")


# ----------------------------------------------------------------------------------
# Array helpers, algebra/array_utils.py:106-136 and :332-367.
# ----------------------------------------------------------------------------------
def neighbour_average(arr, axes):
    """``neighbour_average`` algebra/array_utils.py:106-136 (axes applied in order)."""
    for ax in (axes,) if isinstance(axes, int) else axes:
        i1 = [slice(None)] * arr.ndim
        i2 = [slice(None)] * arr.ndim
        i1[ax] = slice(None, -1)
        i2[ax] = slice(1, None)
        arr = 0.5 * (arr[tuple(i1)] + arr[tuple(i2)])
    return arr


def split_to_vertex(arr, axes):
    """``split_to_vertex`` algebra/array_utils.py:332-367.

    ``jnp.empty`` is zero-filled under JAX, so the first/last vertex along each axis
    receives half of one element and the interior ones ``0.5*a[i] + 0.5*a[i-1]``.
    """
    for ax in (axes,) if isinstance(axes, int) else axes:
        shape = list(arr.shape)
        shape[ax] += 1
        out = np.zeros(shape, REAL)
        i1 = [slice(None)] * len(shape)
        i2 = [slice(None)] * len(shape)
        i1[ax] = slice(None, -1)
        i2[ax] = slice(1, None)
        out[tuple(i1)] = 0.5 * arr
        out[tuple(i2)] += 0.5 * arr
        arr = out
    return arr


def make_rectangular_grid(m, n, chord, ea):
    """``make_rectangular_grid`` aero/utils.py:23-36."""
    grid = np.zeros((m + 1, n + 1, 3))
    grid[..., 0] = (np.linspace(0.0, chord, m + 1) - ea * chord)[:, None]
    return grid


def compute_surf_c(zeta):
    """``compute_surf_c`` aero/utils.py:87-93."""
    return neighbour_average(zeta, (-3, -2))


def compute_surf_nc(zeta):
    """``compute_surf_nc`` aero/utils.py:96-105 (area-length normals)."""
    diag1 = zeta[..., 1:, 1:, :] - zeta[..., :-1, :-1, :]
    diag2 = zeta[..., 1:, :-1, :] - zeta[..., :-1, 1:, :]
    return np.cross(diag1, diag2)


def mirror_grid(zeta, mirror_point, mirror_normal):
    """``mirror_grid`` aero/utils.py:651-663."""
    diff = zeta - mirror_point[None, None, :]
    diff_n = np.einsum("ijk,k->ij", diff, mirror_normal)
    return zeta - 2.0 * diff_n[:, :, None] * mirror_normal[None, None, :]


def chordwise_segments(zeta):
    """Chordwise filaments ``zeta[k,l] -> zeta[k+1,l]``, shape (m, n+1, 2, 3) (aic.py:31, :277)."""
    return np.stack((zeta[:-1, :, :], zeta[1:, :, :]), axis=-2)


def spanwise_segments(zeta):
    """Spanwise filaments ``zeta[k,l] -> zeta[k,l+1]``, shape (m+1, n, 2, 3) (aic.py:34, :280)."""
    return np.stack((zeta[:, :-1, :], zeta[:, 1:, :]), axis=-2)


def gamma_eff(gamma):
    """Filament strengths from ring strengths, aic.py:284-287.

    Chordwise ``G[k,l] - G[k,l-1]`` (m, n+1); spanwise ``G[k-1,l] - G[k,l]`` (m+1, n),
    both zero-padded.
    """
    g_m = np.diff(np.pad(gamma, ((0, 0), (1, 1))), axis=1)
    g_n = -np.diff(np.pad(gamma, ((1, 1), (0, 0))), axis=0)
    return g_m, g_n


# ----------------------------------------------------------------------------------
# Influence sums, aero/aic.py.
# ----------------------------------------------------------------------------------
def _pairwise(kernel, targets, segs, r_cut, reducer):
    """Evaluate ``kernel`` over all (target, segment) pairs in chunks and reduce.

    ``reducer(k_chunk, t0, t1)`` receives kernel values (Tc, S, 3).
    """
    t = targets.reshape(-1, 3)
    s = segs.reshape(-1, 2, 3)
    if s.shape[0] == 0 or t.shape[0] == 0:
        return
    step = max(1, _PAIR_BUDGET // s.shape[0])
    for t0 in range(0, t.shape[0], step):
        t1 = min(t.shape[0], t0 + step)
        k = kernel_eval(kernel, t[t0:t1, None, :], s[None, :, 0, :], s[None, :, 1, :], r_cut)
        reducer(k, t0, t1)


def compute_aic_grid(c, n, zeta, kernel, r_cut=R_CUTOFF):
    """``compute_aic_grid`` aero/aic.py:11-63 with normal projection.

    Returns (c_m, c_n, m, n): influence of every ring of ``zeta`` at each collocation
    point, projected on its (area-length) normal.  Per-segment influences are dotted
    with n_i first and then combined as ``-diff(m_infl, axis=1) + diff(n_infl, axis=0)``.
    """
    c_m, c_n = c.shape[:2]
    m_p, n_p = zeta.shape[0] - 1, zeta.shape[1] - 1
    if not c_m or not c_n or not m_p or not n_p:
        return np.zeros((c_m, c_n, m_p, n_p), REAL)
    cf = c.reshape(-1, 3)
    nf = n.reshape(-1, 3)
    out = np.zeros((cf.shape[0], m_p, n_p), REAL)
    m_segs = chordwise_segments(zeta).reshape(-1, 2, 3)
    n_segs = spanwise_segments(zeta).reshape(-1, 2, 3)
    m_inf = np.zeros((cf.shape[0], m_segs.shape[0]), REAL)
    n_inf = np.zeros((cf.shape[0], n_segs.shape[0]), REAL)

    def red_m(k, t0, t1):
        m_inf[t0:t1] = np.einsum("tsk,tk->ts", k, nf[t0:t1])

    def red_n(k, t0, t1):
        n_inf[t0:t1] = np.einsum("tsk,tk->ts", k, nf[t0:t1])

    _pairwise(kernel, cf, m_segs, r_cut, red_m)
    _pairwise(kernel, cf, n_segs, r_cut, red_n)
    m_inf = m_inf.reshape(-1, m_p, n_p + 1)
    n_inf = n_inf.reshape(-1, m_p + 1, n_p)
    out = -np.diff(m_inf, axis=2) + np.diff(n_inf, axis=1)
    return out.reshape(c_m, c_n, m_p, n_p)


def compute_aic_solve(cs, ns, zetas_b, zetas_w, kernel, mirror=None, r_cut=R_CUTOFF):
    """``compute_aic_solve`` aero/aic.py:137-187 (+ ``compute_aic_sys`` :66-112,
    ``add_wake_influence`` :190-205, ``assemble_aic_sys`` :115-134).

    ``zetas_w`` is given only for the static solve: the influence of every wake ring is
    summed over wake rows onto the trailing-edge (last-row) bound column.
    """

    def sys_mats(zetas):
        mats = []
        for c, n in zip(cs, ns):
            row = []
            for zeta in zetas:
                a = compute_aic_grid(c, n, zeta, kernel, r_cut)
                if mirror is not None:
                    a = a - compute_aic_grid(c, n, mirror_grid(zeta, *mirror), kernel, r_cut)
                row.append(a)
            mats.append(row)
        return mats

    aic_b = sys_mats(zetas_b)
    if zetas_w is not None:
        aic_w = sys_mats(zetas_w)
        for i in range(len(aic_b)):
            for j in range(len(aic_b[i])):
                aic_b[i][j] = aic_b[i][j].copy()
                aic_b[i][j][:, :, -1, :] += np.sum(aic_w[i][j], axis=2)
    rows = []
    for row in aic_b:
        rows.append(
            np.concatenate([a.reshape(a.shape[0] * a.shape[1], a.shape[2] * a.shape[3]) for a in row], axis=1)
        )
    return np.concatenate(rows, axis=0)


def v_ind_segments(targets, segs, g, kernel, r_cut=R_CUTOFF):
    """``v_ind_vmap`` aero/aic.py:208-245: sum_s K(x, seg_s) * g_s for each target."""
    tshape = targets.shape
    t = targets.reshape(-1, 3)
    out = np.zeros_like(t)
    gf = g.ravel()

    def red(k, t0, t1):
        out[t0:t1] = np.einsum("tsk,s->tk", k, gf)

    _pairwise(kernel, t, segs, r_cut, red)
    return out.reshape(tshape)


def compute_v_ind(cs, zetas, gammas, kernel, mirror=None, r_cut=R_CUTOFF):
    """``compute_v_ind`` aero/aic.py:248-310 for one target array ``cs`` (..., 3)."""
    v = np.zeros_like(cs)
    for zeta, gamma in zip(zetas, gammas):
        g_m, g_n = gamma_eff(gamma)
        v = v + (
            v_ind_segments(cs, chordwise_segments(zeta), g_m, kernel, r_cut)
            + v_ind_segments(cs, spanwise_segments(zeta), g_n, kernel, r_cut)
        )
        if mirror is not None:
            zm = mirror_grid(zeta, *mirror)
            v = v - (
                v_ind_segments(cs, chordwise_segments(zm), g_m, kernel, r_cut)
                + v_ind_segments(cs, spanwise_segments(zm), g_n, kernel, r_cut)
            )
    return v


# ----------------------------------------------------------------------------------
# Flow fields, aero/flowfields.py.
# ----------------------------------------------------------------------------------
class Constant:
    """``Constant`` aero/flowfields.py:87-97 (with the base class :13-37)."""

    kind = "constant"

    def __init__(self, u_inf, rho, relative_motion=True):
        self.u_inf = np.asarray(u_inf, dtype=np.float64)
        self.rho = float(rho)
        self.relative_motion = bool(relative_motion)
        self.u_inf_mag = float(np.linalg.norm(self.u_inf))
        self.u_inf_dir = self.u_inf / self.u_inf_mag
        self.q_inf = 0.5 * self.rho * self.u_inf_mag**2

    def __call__(self, x, t):
        out = np.zeros_like(x)
        if self.relative_motion:
            out[...] = self.u_inf
        return out


class OneMinusCosine(Constant):
    """``OneMinusCosine`` aero/flowfields.py:100-181.

    ``0.5*A*(1-cos(pi*s/L))`` for ``0 < s < 2L`` along the travel direction, so the
    reference's ``gust_length`` L is half of the full gust length.
    """

    kind = "one_minus_cosine"

    def __init__(self, u_inf, rho, relative_motion, gust_length, gust_amplitude,
                 gust_travel_direction=None, gust_amplitude_direction=None, gust_x0=None):
        super().__init__(u_inf, rho, relative_motion)
        self.gust_amplitude = float(gust_amplitude)
        self.gust_length = float(gust_length)
        d = self.u_inf_dir if gust_travel_direction is None else np.asarray(gust_travel_direction, float)
        self.gust_travel_direction = d / np.linalg.norm(d)
        a = np.array((0.0, 0.0, 1.0)) if gust_amplitude_direction is None else np.asarray(
            gust_amplitude_direction, float)
        self.gust_amplitude_direction = a / np.linalg.norm(a)
        self.gust_x0 = np.zeros(3) if gust_x0 is None else np.asarray(gust_x0, float)

    def __call__(self, x, t):
        rel_x = x - self.gust_x0
        if self.relative_motion:
            rel_x = rel_x - self.u_inf * t
        gust_x = np.einsum("...k,k->...", rel_x, self.gust_travel_direction)
        val = (self.gust_amplitude_direction * self.gust_amplitude * 0.5
               * (1.0 - np.cos(np.pi * gust_x[..., None] / self.gust_length)))
        inside = ((gust_x > 0) & (gust_x < 2.0 * self.gust_length))[..., None]
        u = np.where(inside, val, 0.0)
        if self.relative_motion:
            u = u + self.u_inf
        return u


# ----------------------------------------------------------------------------------
# Wake, forces and strip angle, aero/utils.py.
# ----------------------------------------------------------------------------------
def _interp(x, xp, fp):
    """np.interp in the arrays' own type: np.interp itself for float64 (the reference's
    jnp.interp semantics as the goldens pin them), the same formula for extended precision
    (np.interp accepts only float64)."""
    if np.result_type(x, xp, fp) == np.float64:
        return np.interp(x, xp, fp)
    out = np.empty(np.shape(x), dtype=REAL)
    last = xp.shape[0] - 1
    for q, xq in enumerate(np.asarray(x)):
        if xq < xp[0]:
            out[q] = fp[0]
        elif xq >= xp[last]:
            out[q] = fp[last]
        else:
            j = int(np.searchsorted(xp, xq, side="right")) - 1
            out[q] = (fp[j + 1] - fp[j]) / (xp[j + 1] - xp[j]) * (xq - xp[j]) + fp[j]
    return out


def propagate_surf_wake(gamma_b_nm1, gamma_w_nm1, zeta_b_n, zeta_w_nm1, delta_w, v_func, dt, arc_held=None,
                        arc_record=None):
    """``propagate_surf_wake`` aero/utils.py:400-500 (uniform and ``delta_w`` branches).
    ``arc_held``: arc lengths to use in place of the convected wake's own (the linear
    model's ``linearise_variable_wake``, whose stop_gradient holds them at the reference
    point, :465-468); ``arc_record``: a list that receives the arc lengths used."""
    zeta_te = zeta_b_n[-1, ...]
    gamma_te = gamma_b_nm1[-1, ...]
    if delta_w is not None:
        zeta_base = zeta_w_nm1
        gamma_base = gamma_w_nm1
    else:
        zeta_base = zeta_w_nm1[:-1, ...]
        gamma_base = gamma_w_nm1[:-1, ...]
    gamma_w_n = np.concatenate((gamma_te[None, ...], gamma_base), axis=0)
    v = v_func(zeta_base)
    zeta_w_n = np.concatenate((zeta_te[None, :, :], zeta_base + dt * v), axis=0)
    if delta_w is not None:
        seg = np.linalg.norm(zeta_w_n[1:, ...] - zeta_w_n[:-1, ...], axis=-1)
        s_zeta_w = np.concatenate((np.zeros((1, zeta_te.shape[0])), np.cumsum(seg, axis=0)), axis=0)
        if arc_held is not None:
            s_zeta_w = np.asarray(arc_held, dtype=s_zeta_w.dtype)
        if arc_record is not None:
            arc_record.append(s_zeta_w.copy())
        s_gamma_w = neighbour_average(s_zeta_w, (0, 1))
        s_disc = np.concatenate((np.zeros(1), np.cumsum(delta_w)))
        s_gamma_disc = neighbour_average(s_disc, (0,))
        zn = np.empty((s_disc.shape[0], zeta_w_n.shape[1], 3), REAL)
        for j in range(zeta_w_n.shape[1]):
            for k in range(3):
                zn[:, j, k] = _interp(s_disc, s_zeta_w[:, j], zeta_w_n[:, j, k])
        gn = np.empty((s_gamma_disc.shape[0], gamma_w_n.shape[1]), REAL)
        for j in range(gamma_w_n.shape[1]):
            gn[:, j] = _interp(s_gamma_disc, s_gamma_w[:, j], gamma_w_n[:, j])
        zeta_w_n, gamma_w_n = zn, gn
    if gamma_w_nm1.size == 0:
        gamma_w_n = np.zeros_like(gamma_w_nm1)
    return zeta_w_n, gamma_w_n


def calculate_steady_forcing(zeta_b, zeta_dot_b, gamma_b, gamma_w, rho, v_func, v_inputs=None):
    """``calculate_steady_forcing`` aero/utils.py:126-223 for a list of surfaces;
    ``v_inputs`` (vertex velocities added at the filament midpoints, :179-181) is the
    linear model's bound upwash."""
    out = []
    v_in = v_inputs if v_inputs is not None else [None] * len(zeta_b)
    for zb, zd, gb, gw, vi in zip(zeta_b, zeta_dot_b, gamma_b, gamma_w, v_in):
        mp_c = neighbour_average(zb, 0)
        mp_s = neighbour_average(zb, 1)
        mpd_c = neighbour_average(zd, 0)
        mpd_s = neighbour_average(zd, 1)
        v_rel_c = v_func(mp_c) - mpd_c
        v_rel_s = v_func(mp_s) - mpd_s
        if vi is not None:
            v_rel_c = v_rel_c + neighbour_average(vi, 0)
            v_rel_s = v_rel_s + neighbour_average(vi, 1)
        g_c = np.zeros(v_rel_c.shape[:-1], REAL)
        g_c[:, :-1] = gb
        g_c[:, 1:] += -gb
        g_s = np.zeros(v_rel_s.shape[:-1], REAL)
        g_s[:-1, :] = -gb
        g_s[1:, :] += gb
        if gw.shape[0] > 0:
            g_s[-1, :] += -gw[0, :]
        r_c = zb[1:, :, :] - zb[:-1, :, :]
        r_s = zb[:, 1:, :] - zb[:, :-1, :]
        f_c = rho * np.einsum("ij,ijk->ijk", g_c, np.cross(v_rel_c, r_c))
        f_s = rho * np.einsum("ij,ijk->ijk", g_s, np.cross(v_rel_s, r_s))
        out.append(split_to_vertex(f_c, 0) + split_to_vertex(f_s, 1))
    return out


def strip_alpha(zeta_b, f_steady, v_func, rho):
    """``strip_alpha`` aero/utils.py:226-273."""
    alphas = []
    for zs, fs in zip(zeta_b, f_steady):
        zle = zs[0, :, :]
        zte = zs[-1, :, :]
        le_j = 0.5 * (zle[:-1, :] + zle[1:, :])
        te_j = 0.5 * (zte[:-1, :] + zte[1:, :])
        c_len = np.linalg.norm(te_j - le_j, axis=-1)
        span_vec = 0.5 * ((zle[1:, :] + zte[1:, :]) - (zle[:-1, :] + zte[:-1, :]))
        b_len = np.linalg.norm(span_vec, axis=-1)
        e_s = span_vec / b_len[:, None]
        strip_mid = 0.5 * (le_j + te_j)
        v_ref = v_func(strip_mid)
        v_mag2 = np.sum(v_ref * v_ref, axis=-1)
        e_l = np.cross(v_ref, e_s)
        e_l = e_l / np.linalg.norm(e_l, axis=-1, keepdims=True)
        f_strip = neighbour_average(fs, 1).sum(axis=0)
        q = 0.5 * rho * v_mag2
        cl = np.sum(f_strip * e_l, axis=-1) / (q * c_len * b_len)
        alphas.append(cl / (2.0 * np.pi))
    return alphas


def apply_polar_correction(zeta_b, f_steady, v_func, rho, polars, alpha):
    """``apply_polar_correction`` aero/utils.py:276-397: per strip of a surface with polars,
    the sectional force q c b (cl e_l + cd e_d) placed at c/4 by triangular chordwise
    weights and split onto the strip's two vertex columns, plus the couple q c b cm e_n as
    opposing leading/trailing-edge forces; cl, cd, cm = polar(alpha).  Returns the corrected
    steady forces and the per-strip lift scale cl / (2 pi alpha) (1 where |2 pi alpha| <=
    EPSILON)."""
    f_out, scale_out = [], []
    for zs, fs, pol, al in zip(zeta_b, f_steady, polars, alpha):
        n = zs.shape[1] - 1
        if pol is None:
            f_out.append(fs)
            scale_out.append(np.ones(n, REAL))
            continue
        m = zs.shape[0] - 1
        if len(pol) != n:
            raise ValueError(f"Expected {n} polar callables, got {len(pol)}")
        zle, zte = zs[0], zs[-1]
        le_j = 0.5 * (zle[:-1] + zle[1:])
        te_j = 0.5 * (zte[:-1] + zte[1:])
        chord = te_j - le_j
        c_len = np.linalg.norm(chord, axis=-1)
        e_c = chord / c_len[:, None]
        span_vec = 0.5 * ((zle[1:] + zte[1:]) - (zle[:-1] + zte[:-1]))
        b_len = np.linalg.norm(span_vec, axis=-1)
        e_s = span_vec / b_len[:, None]
        e_n = np.cross(e_c, e_s)
        e_n = e_n / np.linalg.norm(e_n, axis=-1, keepdims=True)
        v_ref = v_func(0.5 * (le_j + te_j))
        v_mag2 = np.sum(v_ref * v_ref, axis=-1)
        v_mag = np.sqrt(v_mag2)
        q = 0.5 * rho * v_mag2
        e_l = np.cross(v_ref, e_s)
        e_l = e_l / np.linalg.norm(e_l, axis=-1, keepdims=True)
        e_d = v_ref / v_mag[:, None]
        coeffs = [pol[j](al[j]) for j in range(n)]
        cl_p = np.array([cf[0] for cf in coeffs], REAL)
        cd_p = np.array([cf[1] for cf in coeffs], REAL)
        cm_p = np.array([cf[2] for cf in coeffs], REAL)
        cl_uvlm = 2.0 * np.pi * al
        with np.errstate(divide="ignore", invalid="ignore"):
            scale_out.append(np.where(np.abs(cl_uvlm) > EPSILON, cl_p / cl_uvlm, 1.0))
        qcb = q * c_len * b_len
        f_lump = qcb[:, None] * (cl_p[:, None] * e_l + cd_p[:, None] * e_d)
        f_couple = (qcb * cm_p)[:, None] * e_n
        w_chord = np.clip(1.0 - np.abs(np.linspace(0.0, 1.0, m + 1) - 0.25) * m, 0.0, 1.0)
        fc = np.zeros_like(fs)
        lump = 0.5 * w_chord[:, None, None] * f_lump[None]
        fc[:, :-1] += lump
        fc[:, 1:] += lump
        cp = 0.5 * f_couple
        fc[0, :-1] += cp
        fc[0, 1:] += cp
        fc[-1, :-1] -= cp
        fc[-1, 1:] -= cp
        f_out.append(fc)
    return f_out, scale_out


class TabulatedPolar:
    """A strip polar from tables: alpha (ascending, rad) -> (cl, cd, cm) by linear
    interpolation with the end values held outside the table (np.interp)."""

    def __init__(self, alpha, cl, cd, cm):
        self.alpha = np.asarray(alpha, float)
        self.cl, self.cd, self.cm = (np.asarray(v, float) for v in (cl, cd, cm))

    def __call__(self, a):
        return tuple(_interp(np.asarray(a).reshape(1), self.alpha, v)[0] for v in (self.cl, self.cd, self.cm))


def se3_vect_product(hg, x):
    """``se3.vect_product`` algebra/se3.py:209-216 for hg (..., 4, 4), x (..., 3)."""
    return np.einsum("...ij,...j->...i", hg[..., :3, :3], x) + hg[..., :3, 3]


# ----------------------------------------------------------------------------------
# The per-step driver, aero/uvlm.py.
# ----------------------------------------------------------------------------------
@dataclass
class GridDiscretisation:
    """``GridDiscretisation`` aero/data_structures.py:29-40."""

    m: int
    n: int
    m_star: int


@dataclass
class Case:
    """Time-batched solution arrays, one list entry per surface (``AeroCase`` fields,
    aero/data_structures.py:43-615)."""

    zeta_b: list
    zeta_b_dot: list
    zeta_w: list
    c: list
    nc: list
    gamma_b: list
    gamma_b_dot: list
    gamma_w: list
    f_steady: list
    f_unsteady: list
    alpha: list
    t: np.ndarray = field(default=None)


class UVLMRef:
    """FP64 restatement of ``UVLM`` aero/uvlm.py:80-1406 for the configurations the CUDA
    path supports (no control surfaces)."""

    def __init__(self, grid_shapes, dof_mapping, mirror_point=None, mirror_normal=None,
                 kernel=KERNEL_EPSILON, r_cut=R_CUTOFF, free_wake=False,
                 gamma_dot_relaxation=0.7, variable_wake_disc=False, polars=None, polar_circulation_scale=0.0):
        self.grid_disc = [g if isinstance(g, GridDiscretisation) else GridDiscretisation(*g)
                          for g in grid_shapes]
        self.n_surf = len(self.grid_disc)
        if isinstance(dof_mapping, np.ndarray):
            dof_mapping = [dof_mapping]
        self.dof_mapping = [np.asarray(d, dtype=np.int64) for d in dof_mapping]
        if mirror_point is not None:
            mn = np.asarray(mirror_normal, float)
            self.mirror = (np.asarray(mirror_point, float), mn / np.linalg.norm(mn))
        else:
            self.mirror = None
        self.kernel = kernel
        self.r_cut = r_cut
        self.free_wake = free_wake
        self.gamma_dot_relaxation = gamma_dot_relaxation
        self.variable_wake_disc = variable_wake_disc
        # uvlm.py:294-303: per surface None or a sequence of n strip polars
        if polars is None:
            self.polars = [None] * self.n_surf
        else:
            if len(polars) != self.n_surf:
                raise ValueError(f"Expected {self.n_surf} polar entries, got {len(polars)}")
            self.polars = [None if p is None else list(p) for p in polars]
        self.polar_circulation_scale = float(polar_circulation_scale)

    # uvlm.py:387-472
    def set_design_variables(self, dt, flowfield, zeta_b0, hg0, delta_w=None):
        if isinstance(zeta_b0, np.ndarray):
            zeta_b0 = [zeta_b0]
        self.zeta_b0 = [np.asarray(z, REAL) for z in zeta_b0]
        self.hg_ref = np.asarray(hg0, float)
        self.zeta_b_ref = self.hg_to_zeta_b(self.hg_ref)
        self.flowfield = flowfield
        self.dt = float(dt)
        if delta_w is None or isinstance(delta_w, np.ndarray):
            delta_w = [delta_w] * self.n_surf if delta_w is None else [delta_w]
        self.delta_w = list(delta_w)
        self.zeta_w_ref = self.initialise_wake()

    # uvlm.py:537-560
    def hg_to_zeta_b(self, hg_n):
        out = []
        for i in range(self.n_surf):
            this_hg = hg_n[self.dof_mapping[i]]
            out.append(se3_vect_product(this_hg[None, :, :, :], self.zeta_b0[i]))
        return out

    # uvlm.py:562-621 (no control surfaces: the jvp term is zero)
    def hg_dot_to_zeta_b_dot(self, hg_n, hg_dot_n):
        out = []
        for i in range(self.n_surf):
            this_hgd = hg_dot_n[self.dof_mapping[i]]
            out.append(se3_vect_product(this_hgd[None, :, :, :], self.zeta_b0[i]))
        return out

    # uvlm.py:662-689
    def initialise_wake(self, zeta_b=None):
        zeta_b = zeta_b if zeta_b is not None else self.zeta_b_ref
        out = []
        for i, dw in enumerate(self.delta_w):
            zeta_te = zeta_b[i][-1, :, :]
            if dw is None:
                dw = np.ones(self.grid_disc[i].m_star) * self.dt * self.flowfield.u_inf_mag
            grid_s = np.concatenate((np.zeros(1), np.cumsum(dw)))
            out.append(zeta_te[None, :, :] + np.outer(grid_s, self.flowfield.u_inf_dir)[:, None, :])
        return out

    def _horseshoe_wake(self, zeta_b, i):
        """``_make_surf_horseshoe_wake`` uvlm.py:642-660."""
        zeta_te = zeta_b[-1, ...]
        if self.grid_disc[i].m_star == 0:
            return zeta_te[None, :]
        wake_end = zeta_te + (self.flowfield.u_inf_dir * HORSESHOE_LENGTH)[None, :]
        return np.stack((zeta_te, wake_end), axis=0)

    def v_ind(self, x, zetas, gammas):
        return compute_v_ind(x, zetas, gammas, self.kernel, self.mirror, self.r_cut)

    def aic_solve(self, cs, ns, zetas_b, zetas_w):
        return compute_aic_solve(cs, ns, zetas_b, zetas_w, self.kernel, self.mirror, self.r_cut)

    # uvlm.py:824-1117; nu_b / nu_w are the linear model's bound and wake upwash inputs
    # (uvlm.py:943-946, 979-981, and calculate_steady_forcing's v_inputs)
    def base_solve_from_grid(self, q_nm1, t_n, zeta_b_n, zeta_b_nm1, zeta_b_dot_n, static,
                             horseshoe=False, nu_b=None, nu_w=None, arc_held=None, arc_record=None):
        ff = self.flowfield
        c_n = [compute_surf_c(z) for z in zeta_b_n]
        nc_n = [compute_surf_nc(z) for z in zeta_b_n]
        c_dot_n = None if zeta_b_dot_n is None else [neighbour_average(zd, (0, 1)) for zd in zeta_b_dot_n]
        if static:
            if horseshoe:
                zeta_w_n = [self._horseshoe_wake(zeta_b_n[i], i) for i in range(self.n_surf)]
            else:
                zeta_w_n = self.initialise_wake(zeta_b_n)
            gamma_w_n = None
        else:
            gb_nm1, gw_nm1, gbd_nm1, zw_nm1 = q_nm1
            zeta_full = [*zeta_b_nm1, *zw_nm1]
            gamma_full = [*gb_nm1, *gw_nm1]

            def v_wake_prop(x_):
                v = ff(x_, t_n)
                if self.free_wake:
                    v = v + self.v_ind(x_, zeta_full, gamma_full)
                return v

            zeta_w_n, gamma_w_n = [], []
            for i in range(self.n_surf):
                zw, gw = propagate_surf_wake(gb_nm1[i], gw_nm1[i], zeta_b_n[i], zw_nm1[i],
                                             self.delta_w[i], v_wake_prop, self.dt,
                                             None if arc_held is None else arc_held[i], arc_record)
                zeta_w_n.append(zw)
                gamma_w_n.append(gw)
            if nu_w is not None:
                zeta_w_n = [zw + nw * self.dt for zw, nw in zip(zeta_w_n, nu_w)]

        aic = self.aic_solve(c_n, nc_n, zeta_b_n, zeta_w_n if static else None)
        v_bc = [ff(c, t_n) for c in c_n]
        if not static:
            v_bc = [v - cd for v, cd in zip(v_bc, c_dot_n)]
            v_bc = [v + self.v_ind(c, zeta_w_n, gamma_w_n) for v, c in zip(v_bc, c_n)]
        if nu_b is not None:
            v_bc = [v + compute_surf_c(nb) for v, nb in zip(v_bc, nu_b)]
        rhs = np.concatenate([np.einsum("ijk,ijk->ij", v, n).ravel() for v, n in zip(v_bc, nc_n)])
        gamma_vec = _solve(aic, -rhs)
        gamma_b_n, off = [], 0
        for gd in self.grid_disc:
            gamma_b_n.append(gamma_vec[off:off + gd.m * gd.n].reshape(gd.m, gd.n))
            off += gd.m * gd.n
        if static:
            gamma_w_n = [np.broadcast_to(gb[[-1], ...], (1 if (horseshoe and gd.m_star != 0) else gd.m_star, gd.n)).copy()
                         for gb, gd in zip(gamma_b_n, self.grid_disc)]
        zdf = zeta_b_dot_n if zeta_b_dot_n is not None else [np.zeros_like(z) for z in zeta_b_n]

        def v_total(x_):
            return ff(x_, t_n) + self.v_ind(x_, [*zeta_b_n, *zeta_w_n], [*gamma_b_n, *gamma_w_n])

        f_steady = calculate_steady_forcing(zeta_b_n, zdf, gamma_b_n, gamma_w_n, ff.rho, v_total, nu_b)
        alpha_n = strip_alpha(zeta_b_n, f_steady, lambda x_: ff(x_, t_n), ff.rho)
        if any(p is not None for p in self.polars):  # uvlm.py:1055-1075
            f_steady, lift_scale = apply_polar_correction(zeta_b_n, f_steady, lambda x_: ff(x_, t_n), ff.rho,
                                                          self.polars, alpha_n)
            if self.polar_circulation_scale != 0.0:
                sc = self.polar_circulation_scale
                gamma_b_n = [gb * (1.0 + sc * (ls[None, :] - 1.0)) for gb, ls in zip(gamma_b_n, lift_scale)]
                if static:
                    gamma_w_n = [np.broadcast_to(gb[[-1], ...], gw.shape).copy()
                                 for gb, gw in zip(gamma_b_n, gamma_w_n)]
        if static:
            gamma_b_dot_n = None
            f_unsteady = None
        else:
            g = self.gamma_dot_relaxation
            gamma_b_dot_n = [(gb - gbm) / self.dt * g + gbd * (1.0 - g)
                             for gb, gbm, gbd in zip(gamma_b_n, gb_nm1, gbd_nm1)]
            f_unsteady = [split_to_vertex(ff.rho * gbd[..., None] * nc, (0, 1))
                          for gbd, nc in zip(gamma_b_dot_n, nc_n)]
        return dict(c=c_n, nc=nc_n, gamma_b=gamma_b_n, gamma_w=gamma_w_n, gamma_b_dot=gamma_b_dot_n,
                    zeta_b=zeta_b_n, zeta_w=zeta_w_n, zeta_b_dot=zeta_b_dot_n, f_steady=f_steady,
                    f_unsteady=f_unsteady, alpha=alpha_n)

    def _empty_case(self, n_tstep):
        """``initialise_case_object`` uvlm.py:1217-1284 (zero-filled)."""
        gds = self.grid_disc
        return Case(
            zeta_b=[np.zeros((n_tstep, g.m + 1, g.n + 1, 3), REAL) for g in gds],
            zeta_b_dot=[np.zeros((n_tstep, g.m + 1, g.n + 1, 3), REAL) for g in gds],
            zeta_w=[np.zeros((n_tstep, g.m_star + 1, g.n + 1, 3), REAL) for g in gds],
            c=[np.zeros((n_tstep, g.m, g.n, 3), REAL) for g in gds],
            nc=[np.zeros((n_tstep, g.m, g.n, 3), REAL) for g in gds],
            gamma_b=[np.zeros((n_tstep, g.m, g.n), REAL) for g in gds],
            gamma_b_dot=[np.zeros((n_tstep, g.m, g.n), REAL) for g in gds],
            gamma_w=[np.zeros((n_tstep, g.m_star, g.n), REAL) for g in gds],
            f_steady=[np.zeros((n_tstep, g.m + 1, g.n + 1, 3), REAL) for g in gds],
            f_unsteady=[np.zeros((n_tstep, g.m + 1, g.n + 1, 3), REAL) for g in gds],
            alpha=[np.zeros((n_tstep, g.n), REAL) for g in gds],
            t=np.zeros(n_tstep, REAL),
        )

    @staticmethod
    def _store(case, i_ts, out, static):
        """``case_solve`` uvlm.py:1188-1213."""
        for key in ("c", "nc", "gamma_b", "gamma_w", "zeta_b", "f_steady", "alpha", "zeta_w"):
            for arr, val in zip(getattr(case, key), out[key]):
                arr[i_ts] = val
        if not static:
            for key in ("gamma_b_dot", "zeta_b_dot", "f_unsteady"):
                for arr, val in zip(getattr(case, key), out[key]):
                    arr[i_ts] = val

    # uvlm.py:1286-1333
    def solve_static(self, hg=None, t=0.0, horseshoe=False):
        case = self._empty_case(1)
        case.t[0] = t
        hg_n = hg if hg is not None else self.hg_ref
        out = self.base_solve_from_grid(None, t, self.hg_to_zeta_b(hg_n), None, None, True, horseshoe)
        if horseshoe:
            out["zeta_w"] = self.initialise_wake(out["zeta_w"])
        self._store(case, 0, out, True)
        if horseshoe:
            for i, zw in enumerate(self.initialise_wake(zeta_b=[z[0] for z in case.zeta_b])):
                case.zeta_w[i][0] = zw
        return case

    # uvlm.py:1335-1406 with case_solve uvlm.py:1119-1215
    def solve_prescribed_dynamic(self, init_case, hg_t, hg_dot_t, n_steps=None):
        n_tstep = hg_t.shape[0]
        case = self._empty_case(n_tstep)
        for key in ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w",
                    "f_steady", "f_unsteady", "alpha"):
            for arr, val in zip(getattr(case, key), getattr(init_case, key)):
                arr[0] = val[0]
        case.t[0] = init_case.t[0]
        last = n_tstep if n_steps is None else min(n_tstep, n_steps + 1)
        for i in range(1, last):
            self.case_step(case, i, hg_t[i], hg_t[i - 1], hg_dot_t[i])
        return case

    def case_step(self, case, i, hg_n, hg_nm1, hg_dot_n):
        """One dynamic ``case_solve`` (uvlm.py:1119-1215)."""
        q_nm1 = ([g[i - 1] for g in case.gamma_b], [g[i - 1] for g in case.gamma_w],
                 [g[i - 1] for g in case.gamma_b_dot], [z[i - 1] for z in case.zeta_w])
        case.t[i] = case.t[i - 1] + self.dt
        out = self.base_solve_from_grid(
            q_nm1, case.t[i], self.hg_to_zeta_b(hg_n), self.hg_to_zeta_b(hg_nm1),
            self.hg_dot_to_zeta_b_dot(hg_n, hg_dot_n), False)
        self._store(case, i, out, False)
        return case


def force_coefficients(case, flowfield, s_ref, alpha_deg):
    """CL, CD per time step from the summed vertex forces ``f_steady + f_unsteady``.

    Lift and drag axes are ``e_L = (-sin a, 0, cos a)`` and ``e_D = (cos a, 0, sin a)``
    (the convention of tests/aero/test_infinite_wing_polar.py:92, :161); ``q = 0.5 rho |U|^2``.
    """
    a = np.deg2rad(alpha_deg)
    e_l = np.array((-np.sin(a), 0.0, np.cos(a)))
    e_d = np.array((np.cos(a), 0.0, np.sin(a)))
    f = sum(fs.sum(axis=(1, 2)) + fu.sum(axis=(1, 2)) for fs, fu in zip(case.f_steady, case.f_unsteady))
    q = flowfield.q_inf * s_ref
    return f @ e_l / q, f @ e_d / q
