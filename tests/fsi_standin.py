"""A stand-in structure for fluid-structure loops in tests (TEST INFRASTRUCTURE).

The reference couples the UVLM to its geometrically exact beam inside
``fsi_convergence_loop`` (structure/beam.py:2612-2697): per time step it repeatedly builds
the node frames hg_n and their rates from the current structural guess, calls
``aero_obj.case_solve(case, i_ts, hg_n, hg_nm1, hg_dot_n, static=False, horseshoe=False,
...)``, projects the solved slot onto the nodes with
``aero_sol.project_forcing_to_beam(i_ts, rmat=hg_n[:, :3, :3], x0_aero=aero_obj.zeta_b0,
include_unsteady=aero_obj.include_unsteady_force)`` and updates the structure with those
loads.  ``run_fsi`` is that loop with the beam replaced by a rigid wing on heave and pitch
springs (a typical section), integrated by the average-acceleration Newmark rule, and a
fixed number of iterations per step.  The same function drives the reference's own UVLM
(through the NumPy stand-in for jax, to make golden vectors) and this package's UVLM.
"""
from __future__ import annotations

import numpy as np


class TypicalSection:
    """Heave h (z, up) and pitch theta (about y through the node line, nose up) of a rigid
    wing whose nodes sit on the y axis; m h'' + k_h h = sum F_z, I theta'' + k_t theta =
    sum M_y of the projected loads."""

    def __init__(self, y_nodes, mass=200.0, k_heave=200.0, inertia=50.0, k_pitch=100.0):
        self.y = np.asarray(y_nodes, float)
        self.m = np.array([mass, inertia])
        self.k = np.array([k_heave, k_pitch])

    def frames(self, x, v):
        """hg (n_nodes, 4, 4) and its rate for generalised coordinates x = (h, theta) and
        rates v."""
        h, th = x
        hd, thd = v
        c, s = np.cos(th), np.sin(th)
        n = self.y.size
        hg = np.zeros((n, 4, 4))
        hg[:, :3, :3] = np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])
        hg[:, 1, 3] = self.y
        hg[:, 2, 3] = h
        hg[:, 3, 3] = 1.0
        hgd = np.zeros((n, 4, 4))
        hgd[:, :3, :3] = thd * np.array([[-s, 0.0, c], [0.0, 0.0, 0.0], [-c, 0.0, -s]])
        hgd[:, 2, 3] = hd
        return hg, hgd

    @staticmethod
    def loads(f_proj):
        """Generalised forces (sum of F_z, sum of M_y) from projected node loads (n, 6)."""
        return np.array([f_proj[:, 2].sum(), f_proj[:, 4].sum()])

    def newmark(self, x, v, a, f, dt):
        """Average-acceleration Newmark step of the two decoupled oscillators."""
        a1 = (f - self.k * (x + dt * v + 0.25 * dt * dt * a)) / (self.m + 0.25 * dt * dt * self.k)
        v1 = v + 0.5 * dt * (a + a1)
        x1 = x + dt * v + 0.25 * dt * dt * (a + a1)
        return x1, v1, a1


def run_fsi(uvlm, struct: TypicalSection, init_case, n_tstep, dt, n_iter=3, record=None):
    """Time-march a UVLM (the reference's or this package's: anything with the reference's
    ``case_solve`` / ``project_forcing_to_beam`` surface) coupled to ``struct``.

    ``init_case`` is a batched AeroCase whose slot 0 holds the static solution at the
    undeformed frames.  ``record`` (a list) receives, per time step and iterate,
    ``(i_ts, iterate, hg_n, hg_dot_n, f_proj)``.  Returns the case and the structural
    history (x, v, a), each ``(n_tstep, 2)``.
    """
    x = np.zeros((n_tstep, 2))
    v = np.zeros((n_tstep, 2))
    a = np.zeros((n_tstep, 2))
    hg_prev, _ = struct.frames(x[0], v[0])
    f_prev = struct.loads(init_case.project_forcing_to_beam(0, hg_prev[:, :3, :3], uvlm.zeta_b0,
                                                            uvlm.include_unsteady_force))
    # start at rest at the static loads' equilibrium acceleration
    a[0] = (f_prev - struct.k * x[0]) / struct.m
    case = init_case
    for i in range(1, n_tstep):
        f = f_prev
        for it in range(n_iter):
            xi, vi, ai = struct.newmark(x[i - 1], v[i - 1], a[i - 1], f, dt)
            hg_n, hgd_n = struct.frames(xi, vi)
            case = uvlm.case_solve(case=case, i_ts=i, hg_n=hg_n, hg_nm1=hg_prev, hg_dot_n=hgd_n, static=False,
                                   horseshoe=False, cs_ang_n={}, cs_ang_nm1={}, cs_vel_n={})
            fp = np.asarray(case.project_forcing_to_beam(i, hg_n[:, :3, :3], uvlm.zeta_b0,
                                                         uvlm.include_unsteady_force))
            if record is not None:
                record.append((i, it, hg_n, hgd_n, fp))
            f = struct.loads(fp)
        x[i], v[i], a[i] = xi, vi, ai
        hg_prev = hg_n
        f_prev = f
    return case, (x, v, a)
