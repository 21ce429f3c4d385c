"""CPU restatement of ``UVLM.timestep_residual`` (aero/uvlm.py:1942-2047) for checking the
CUDA-backed residual VJP.  Test infrastructure: only tests import this module.

The reference takes beam coordinates (varphi, v) and maps them to node frames through
beam code (``calculate_hg_from_varphi``, ``make_hg_dot``); here the frames hg_n,
hg_dot_n, hg_nm1 are the inputs, and everything from the frames on follows the
reference:

* r_gamma_b = solve(A_n, -(u - c_dot + V_w(c; zeta_w_n, gamma_w_n)) . n) - gamma_b_n
  (``gamma_b_res_func`` :1529-1645);
* r_gamma_w, r_zeta_w = propagate_wake(q_{n-1}, zeta_b_n) - (gamma_w_n, zeta_w_n), the free
  wake convected by the lattices of n-1 (``wake_prop_res_func`` :1647-1751);
* r_gamma_dot = g/dt (gamma_b_n - gamma_b_{n-1}) + (1-g) gamma_dot_{n-1} - gamma_dot_n
  (``gamma_b_dot_res_func`` :1753-1801);
* r_f = R^T project_forcing_to_beam(f_steady + f_unsteady) - f_beam_n, the forces from the
  states of step n (``f_aero_res_func`` :1803-1940; ``project_forcing_to_beam``
  aero/utils.py:666-697; ``transform_nodal_vect`` structure/utils.py:249-260).

States per surface: gamma_b (m, n), gamma_w (m_star, n), gamma_b_dot (m, n), zeta_w
(m_star+1, n+1, 3), as dicts of lists.  The residual is returned as the reference's
concatenation [r_gamma_b, r_gamma_w, r_gamma_dot, r_zeta_w, r_f].
"""
from __future__ import annotations

import numpy as np

from oracle import uvlm_ref as R


def project_forcing_to_beam(f_total, rmat, dof_mapping, x0_aero):
    """aero/utils.py:666-697: per node the strip's summed force and the moment of the forces
    about the node (arms R x0); nodes written in surface order (a node shared by two vertex
    columns keeps the last one, as the reference's scatter-set with unique indices)."""
    out = np.zeros((rmat.shape[0], 6), dtype=np.result_type(rmat, f_total[0]))
    for f, dof, x0 in zip(f_total, dof_mapping, x0_aero):
        r_x0 = np.einsum("ijk,lik->lij", rmat[dof], x0)  # (m+1, n+1, 3)
        out[dof, :3] = f.sum(axis=0)
        out[dof, 3:] = np.cross(r_x0, f).sum(axis=0)
    return out


def transform_nodal_vect(vect, rmat):
    """structure/utils.py:249-260: both 3-vectors of every node rotated by rmat."""
    return np.concatenate([np.einsum("...ijk,...ik->...ij", rmat, vect[..., :3]),
                           np.einsum("...ijk,...ik->...ij", rmat, vect[..., 3:])], axis=-1)


def timestep_residual(ref, t_n, hg_n, hg_dot_n, hg_nm1, q_n, q_nm1, f_beam_n, include_unsteady=True):
    ff = ref.flowfield
    S = ref.n_surf
    zb = ref.hg_to_zeta_b(hg_n)
    zb_nm1 = ref.hg_to_zeta_b(hg_nm1)
    zbd = ref.hg_dot_to_zeta_b_dot(hg_n, hg_dot_n)
    c = [R.compute_surf_c(z) for z in zb]
    nc = [R.compute_surf_nc(z) for z in zb]
    cdot = [R.neighbour_average(z, (0, 1)) for z in zbd]
    gb, gw, gbd, zw = q_n["gamma_b"], q_n["gamma_w"], q_n["gamma_b_dot"], q_n["zeta_w"]
    gb1, gw1, gbd1, zw1 = q_nm1["gamma_b"], q_nm1["gamma_w"], q_nm1["gamma_b_dot"], q_nm1["zeta_w"]
    # bound circulation
    aic = ref.aic_solve(c, nc, zb, None)
    v_bc = [ff(ci, t_n) - cd + ref.v_ind(ci, zw, gw) for ci, cd in zip(c, cdot)]
    rhs = np.concatenate([np.einsum("ijk,ijk->ij", v, n).ravel() for v, n in zip(v_bc, nc)])
    x = R._solve(aic, -rhs)
    r_gb, off = [], 0
    for s in range(S):
        k = gb[s].size
        r_gb.append(x[off:off + k].reshape(gb[s].shape) - gb[s])
        off += k

    # wake
    def v_prop(x_):
        v = ff(x_, t_n)
        if ref.free_wake:
            v = v + ref.v_ind(x_, [*zb_nm1, *zw1], [*gb1, *gw1])
        return v

    r_zw, r_gw = [], []
    for s in range(S):
        z_new, g_new = R.propagate_surf_wake(gb1[s], gw1[s], zb[s], zw1[s], ref.delta_w[s], v_prop, ref.dt)
        r_zw.append(z_new - zw[s])
        r_gw.append(g_new - gw[s])
    # gamma_dot
    g = ref.gamma_dot_relaxation
    r_gbd = [g / ref.dt * (a - b) + (1.0 - g) * d1 - d for a, b, d1, d in zip(gb, gb1, gbd1, gbd)]

    # forces from the states of step n
    def v_total(x_):
        return ff(x_, t_n) + ref.v_ind(x_, [*zb, *zw], [*gb, *gw])

    fs = R.calculate_steady_forcing(zb, zbd, gb, gw, ff.rho, v_total)
    ft = [f + R.split_to_vertex(ff.rho * d[..., None] * n, (0, 1)) for f, d, n in zip(fs, gbd, nc)] \
        if include_unsteady else fs
    rm = hg_n[:, :3, :3]
    f_glob = project_forcing_to_beam(ft, rm, ref.dof_mapping, ref.zeta_b0)
    r_f = transform_nodal_vect(f_glob, np.swapaxes(rm, -2, -1)) - f_beam_n
    return np.concatenate([np.concatenate([a.ravel() for a in r_gb]), np.concatenate([a.ravel() for a in r_gw]),
                           np.concatenate([a.ravel() for a in r_gbd]), np.concatenate([a.ravel() for a in r_zw]),
                           r_f.ravel()])
