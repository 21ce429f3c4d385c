"""Seeded synthetic UVLM workloads.

Every input is generated here from ``numpy.random.default_rng(seed)``; there is no
dataset.  The rectangular wing, node frames and motion histories follow the patterns of
the reference's own tests (tests/aero/test_mirrored_wing.py:30-35 for the frames,
tests/aero/test_variable_wake_disc.py:41-55 for heave, test_linear_planar_wing.py:146-171
for pitch).

Workloads (chord c = 1, span b = 8, freestream |U| = 1, rho = 1.225, dt = c / (M |U|)):
  wing_heave   8 x 32, W = 64, prescribed wake, epsilon kernel, 5 deg AoA, heave
               0.05 c at reduced frequency 0.2, 50 steps
  wing_free    16 x 128, W = 200, free wake, cutoff kernel (core radius 1e-3 c), linear
               twist (tip angle ~ U[-3, 3] deg), NACA 4-digit camber (max camber
               ~ U[0, 0.04] at 40 % chord), 5 deg AoA, static wing, 200 steps
  wing_pitch   12 x 64, W = 100, 32 twist control points ~ N(0, 1 deg) interpolated to
               the 65 stations, pitch 2 deg at reduced frequency 0.3, 1000 steps
  serving      M ~ U{4..16}, N ~ U{16..128}, W ~ U{20..200}, AoA ~ U[0, 8] deg, heave,
               100 steps per case
All start from the static solution (``solve_static``) of the undeformed wing.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class WingCase:
    name: str
    m: int
    n: int
    m_star: int
    n_steps: int
    chord: float
    span: float
    alpha_deg: float
    u_mag: float
    rho: float
    dt: float
    zeta_b0: np.ndarray       # (m+1, n+1, 3)
    hg0: np.ndarray           # (n+1, 4, 4)
    hg_t: np.ndarray          # (n_steps+1, n+1, 4, 4)
    hg_dot_t: np.ndarray
    free_wake: bool
    kernel: str               # "epsilon" | "cutoff"
    r_cut: float
    seed: int
    extra: dict = field(default_factory=dict)

    @property
    def n_tstep(self):
        return self.n_steps + 1

    @property
    def u_inf(self):
        a = np.deg2rad(self.alpha_deg)
        return self.u_mag * np.array((np.cos(a), 0.0, np.sin(a)))

    @property
    def s_ref(self):
        return self.chord * self.span

    def pairs_per_step(self, mirror=False):
        """(target, filament) kernel evaluations in one dynamic step of the reference
        (AIC + wake RHS + force midpoints + free-wake convection)."""
        m, n, w = self.m, self.n, self.m_star
        nb = m * n
        sb = m * (n + 1) + (m + 1) * n
        sw = w * (n + 1) + (w + 1) * n
        pairs = nb * sb + nb * sw + sb * (sb + sw)
        if self.free_wake:
            pairs += w * (n + 1) * (sb + sw)
        return pairs * (2 if mirror else 1)


def frames(n_nodes: int, span: float, y0: float = 0.0) -> np.ndarray:
    """Identity node frames on the y axis from y0 to y0 + span."""
    hg = np.zeros((n_nodes, 4, 4))
    hg[:, :3, :3] = np.eye(3)
    hg[:, 1, 3] = np.linspace(y0, y0 + span, n_nodes)
    hg[:, 3, 3] = 1.0
    return hg


def naca_camber(xc: np.ndarray, m_c: float, p: float = 0.4) -> np.ndarray:
    """NACA 4-digit mean line z/c at chord fractions xc."""
    return np.where(xc < p, m_c / p**2 * (2 * p * xc - xc**2),
                    m_c / (1 - p)**2 * ((1 - 2 * p) + 2 * p * xc - xc**2))


def twisted_grid(m, n, chord, ea, twist_rad, camber=0.0):
    """Rectangular grid with camber, each spanwise station rotated about the local y
    axis through the elastic axis by ``twist_rad[j]`` (positive nose up)."""
    g = np.zeros((m + 1, n + 1, 3))
    xc = np.linspace(0.0, 1.0, m + 1)
    x = (xc - ea) * chord
    z = naca_camber(xc, camber) * chord if camber else np.zeros_like(xc)
    for j in range(n + 1):
        th = twist_rad[j]
        c, s = np.cos(th), np.sin(th)
        g[:, j, 0] = c * x + s * z
        g[:, j, 2] = -s * x + c * z
    return g


def heave_motion(hg0, n_steps, dt, amp, omega):
    t = np.arange(n_steps + 1) * dt
    hg_t = np.repeat(hg0[None], n_steps + 1, axis=0)
    hg_t[:, :, 2, 3] += (amp * np.sin(omega * t))[:, None]
    hg_dot_t = np.zeros_like(hg_t)
    hg_dot_t[:, :, 2, 3] = (amp * omega * np.cos(omega * t))[:, None]
    return hg_t, hg_dot_t


def pitch_motion(hg0, n_steps, dt, amp, omega):
    """Pitch about each node's y axis (the node frame origin is on the elastic axis);
    hg_dot is the skew rate matrix, as tests/aero/test_linear_planar_wing.py:158-171."""
    t = np.arange(n_steps + 1) * dt
    a = amp * np.sin(omega * t)
    ad = amp * omega * np.cos(omega * t)
    hg_t = np.repeat(hg0[None], n_steps + 1, axis=0)
    c, s = np.cos(a), np.sin(a)
    rot = np.zeros((n_steps + 1, 3, 3))
    rot[:, 0, 0] = c
    rot[:, 0, 2] = s
    rot[:, 1, 1] = 1.0
    rot[:, 2, 0] = -s
    rot[:, 2, 2] = c
    hg_t[:, :, :3, :3] = rot[:, None]
    hg_dot_t = np.zeros_like(hg_t)
    hg_dot_t[:, :, 0, 2] = ad[:, None]
    hg_dot_t[:, :, 2, 0] = -ad[:, None]
    return hg_t, hg_dot_t


def wing_heave(m=8, n=32, m_star=64, n_steps=50, span=8.0, alpha_deg=5.0, k=0.2, amp=0.05, seed=0) -> WingCase:
    chord, u = 1.0, 1.0
    dt = chord / (m * u)
    zeta = np.zeros((m + 1, n + 1, 3))
    zeta[..., 0] = (np.linspace(0.0, chord, m + 1) - 0.25 * chord)[:, None]
    hg0 = frames(n + 1, span)
    omega = 2.0 * k * u / chord
    hg_t, hg_dot_t = heave_motion(hg0, n_steps, dt, amp * chord, omega)
    return WingCase("wing_heave", m, n, m_star, n_steps, chord, span, alpha_deg, u, 1.225, dt, zeta, hg0, hg_t,
                    hg_dot_t, False, "epsilon", 1e-4, seed, dict(k=k, amp=amp))


def wing_free(m=16, n=128, m_star=200, n_steps=200, span=8.0, alpha_deg=5.0, r_core=1e-3, seed=0) -> WingCase:
    rng = np.random.default_rng(seed)
    chord, u = 1.0, 1.0
    dt = chord / (m * u)
    tip = np.deg2rad(rng.uniform(-3.0, 3.0))
    camber = rng.uniform(0.0, 0.04)
    y = np.linspace(0.0, span, n + 1)
    zeta = twisted_grid(m, n, chord, 0.25, tip * y / span, camber)
    hg0 = frames(n + 1, span)
    hg_t = np.repeat(hg0[None], n_steps + 1, axis=0)
    hg_dot_t = np.zeros_like(hg_t)
    return WingCase("wing_free", m, n, m_star, n_steps, chord, span, alpha_deg, u, 1.225, dt, zeta, hg0, hg_t,
                    hg_dot_t, True, "cutoff", r_core * chord, seed, dict(tip_twist_rad=tip, max_camber=camber))


def wing_pitch(m=12, n=64, m_star=100, n_steps=1000, span=8.0, alpha_deg=5.0, k=0.3, amp_deg=2.0, n_ctrl=32,
               seed=0) -> WingCase:
    rng = np.random.default_rng(seed)
    chord, u = 1.0, 1.0
    dt = chord / (m * u)
    ctrl = np.deg2rad(rng.normal(0.0, 1.0, n_ctrl))
    y = np.linspace(0.0, span, n + 1)
    twist = np.interp(y, np.linspace(0.0, span, n_ctrl), ctrl)
    zeta = twisted_grid(m, n, chord, 0.25, twist)
    hg0 = frames(n + 1, span)
    omega = 2.0 * k * u / chord
    hg_t, hg_dot_t = pitch_motion(hg0, n_steps, dt, np.deg2rad(amp_deg), omega)
    return WingCase("wing_pitch", m, n, m_star, n_steps, chord, span, alpha_deg, u, 1.225, dt, zeta, hg0, hg_t,
                    hg_dot_t, False, "epsilon", 1e-4, seed, dict(twist_ctrl_rad=ctrl, k=k, amp_deg=amp_deg))


def serving_stream(n_cases=512, rate=200.0, n_steps=100, seed=0):
    """Case list and Poisson arrival times for the serving workload."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_cases))
    cases = []
    for i in range(n_cases):
        m = int(rng.integers(4, 17))
        n = int(rng.integers(16, 129))
        w = int(rng.integers(20, 201))
        a = float(rng.uniform(0.0, 8.0))
        c = wing_heave(m=m, n=n, m_star=w, n_steps=n_steps, alpha_deg=a, seed=seed * 100003 + i)
        c.name = f"serving_{i}"
        cases.append(c)
    return cases, arrivals


def build_uvlm(case: WingCase, uvlm_cls, flowfield_cls, kernels, grid_cls, precision="fp64", **kw):
    """Construct and configure a UVLM object of either implementation for a WingCase.

    ``kernels`` maps "epsilon"/"cutoff" to that implementation's kernel selector; for the
    cutoff kernel with a non-default radius pass a factory under "cutoff_radius".
    """
    if case.kernel == "cutoff" and "cutoff_radius" in kernels:
        kernel = kernels["cutoff_radius"](case.r_cut)
    else:
        kernel = kernels[case.kernel]
    args = dict(grid_shapes=[grid_cls(case.m, case.n, case.m_star)], dof_mapping=np.arange(case.n + 1),
                kernel=kernel, free_wake=case.free_wake)
    if precision is not None:
        args["precision"] = precision
    args.update(kw)
    uv = uvlm_cls(**args)
    ff = flowfield_cls(case.u_inf, case.rho, True)
    uv.set_design_variables(dt=case.dt, flowfield=ff, zeta_b0=case.zeta_b0, hg0=case.hg0)
    return uv, ff
