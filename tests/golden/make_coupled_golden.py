"""Golden vectors of the reference's own coupled aeroelastic loop (TEST INFRASTRUCTURE).

Runs FLAPJAX's geometrically exact beam (structure/beam.py) coupled to its UVLM
(coupled/coupled.py:161-305 static, :307-434 dynamic) through the NumPy stand-in for jax
in ``jaxshim/`` -- forward derivatives (jax.jvp at algebra/se3.py:389 and beam.py:780,
jax.jacobian at structure/utils.py:76, 179, 221) become central differences there, which
changes only the beam's tangent matrices and damping terms at ~1e-10.  Every
``UVLM.case_solve`` call of the beam's FSI iterations (beam.py:2656-2674) is recorded with
its frames and the loads that ``project_forcing_to_beam`` hands back to the beam, so that a
test can replay the same call sequence through flapjax_b200.UVLM.

The case is the coupled workload in small: a clamped cantilever wing (EA 1e7, GJ = EI =
1e4) on a beam along y, mirrored about y = 0, with a free wake, in a 1-cos vertical gust of
amplitude 0.05 |U| and length 10 c that starts to reach the wing at t = 0.  Its mass, 3
per unit span, is four times the workload's 0.75: with 0.75 the wing is lighter than the
air it moves (rho pi c^2 / 4 = 0.96 per unit span), and the beam's fixed-point FSI
iteration (no relaxation in the dynamic loop) diverges within the first step.  The kernel
is the cutoff one because the beam's converged frames of step n-1 differ from those of its
last aero call by ~6e-6, so the first wake row sits ~6e-6 from the trailing edge it was
shed from, and the epsilon kernel evaluates those pairs near its regularised peak (single
terms ~1e4 times the convection velocity); a vortex core cuts them.

    FLAPJAX_REF_SRC=<reference>/src python tests/golden/make_coupled_golden.py
writes tests/golden/fsi/coupled_beam_gust.npz (a few minutes on one core).
"""
from __future__ import annotations

import importlib
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import make_golden as MG  # noqa: E402

OUT = HERE / "fsi" / "coupled_beam_gust.npz"
N_NODES, M, M_STAR, N_TSTEP = 9, 4, 8, 7
SPAN, CHORD, EA_FRAC = 8.0, 1.0, 0.25
U_INF = np.array((5.0, 0.0, 0.5))
RHO = 1.225
K_CS = np.diag((1e7, 1e7, 1e7, 1e4, 1e4, 1e4))
M_CS = np.diag((3.0, 3.0, 3.0, 0.4, 0.2, 0.2))
GUST_LENGTH, GUST_AMP = 5.0 * CHORD, 0.05 * float(np.linalg.norm(U_INF))  # half length L (full gust 2L)
GUST_X0 = np.array((-10.0, 0.0, 0.0))
R_CORE = 1e-3 * CHORD
FIELDS = ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
          "f_unsteady", "alpha")


def load_coupled():
    ref = MG.load_reference()
    for pkg in ("flapjax.coupled", "flapjax.structure"):
        sys.modules.pop(pkg, None)
    for pkg in ("flapjax.structure", "flapjax.coupled"):
        importlib.import_module(pkg)
    from flapjax.aero.flowfields import OneMinusCosine
    from flapjax.aero.utils import make_rectangular_grid
    from flapjax.coupled import CoupledAeroelastic
    from flapjax.structure import BeamStructure

    ref.OneMinusCosine = OneMinusCosine
    ref.make_rectangular_grid = make_rectangular_grid
    ref.CoupledAeroelastic = CoupledAeroelastic
    ref.BeamStructure = BeamStructure
    return ref


def main():
    ref = load_coupled()
    jnp = ref.jnp
    n = N_NODES - 1
    conn = np.stack([np.arange(n), np.arange(1, N_NODES)], axis=1)
    beam = ref.BeamStructure(num_nodes=N_NODES, connectivity=jnp.array(conn), y_vector=jnp.array((0.0, 0.0, 1.0)))
    ref.utils.R_CUTOFF = R_CORE  # module constant read by biot_savart_cutoff (aero/utils.py:648)
    uvlm = ref.UVLM(grid_shapes=[ref.GridDiscretisation(M, n, M_STAR)], dof_mapping=jnp.arange(N_NODES),
                    mirror_point=jnp.zeros(3), mirror_normal=jnp.array((0.0, 1.0, 0.0)), free_wake=True,
                    kernel=ref.utils.biot_savart_cutoff)
    wing = ref.CoupledAeroelastic(beam, uvlm)
    coords = np.zeros((N_NODES, 3))
    coords[:, 1] = np.linspace(0.0, SPAN, N_NODES)
    dt = CHORD / (np.linalg.norm(U_INF) * M)
    flow = ref.OneMinusCosine(u_inf=jnp.array(U_INF), rho=RHO, relative_motion=True, gust_length=GUST_LENGTH,
                              gust_amplitude=GUST_AMP, gust_x0=jnp.array(GUST_X0))
    grid = ref.make_rectangular_grid(M, n, CHORD, EA_FRAC)
    wing.set_design_variables(coords=jnp.array(coords), k_cs=jnp.array(K_CS), m_cs=jnp.array(M_CS), m_lumped=None,
                              dt=float(dt), flowfield=flow, x0_aero=grid, delta_w=None)

    t0 = time.time()
    static = wing.static_solve(prescribed_dofs=tuple(range(6)), horseshoe=False)
    print(f"static {time.time() - t0:.1f} s", flush=True)

    rec = {"i": [], "hg_n": [], "hg_nm1": [], "hg_dot_n": [], "f": []}
    init = {}
    inner = uvlm.case_solve

    def recording_case_solve(case, i_ts, hg_n, hg_nm1, hg_dot_n, static, horseshoe, cs_ang_n=None,
                             cs_ang_nm1=None, cs_vel_n=None):
        if not init:
            snap = case[0]
            for k in FIELDS:
                init[k] = np.asarray(getattr(snap, k)[0], float)
            init["t"] = float(np.asarray(case.t)[0])
        out = inner(case=case, i_ts=i_ts, hg_n=hg_n, hg_nm1=hg_nm1, hg_dot_n=hg_dot_n, static=static,
                    horseshoe=horseshoe, cs_ang_n=cs_ang_n, cs_ang_nm1=cs_ang_nm1, cs_vel_n=cs_vel_n)
        f = out.project_forcing_to_beam(i_ts=i_ts, rmat=hg_n[:, :3, :3], x0_aero=uvlm.zeta_b0,
                                        include_unsteady=uvlm.include_unsteady_force)
        rec["i"].append(int(i_ts))
        rec["hg_n"].append(np.asarray(hg_n, float))
        rec["hg_nm1"].append(np.asarray(hg_nm1, float))
        rec["hg_dot_n"].append(np.asarray(hg_dot_n, float))
        rec["f"].append(np.asarray(f, float))
        return out

    uvlm.case_solve = recording_case_solve
    dyn = wing.dynamic_solve(init_case=static, prescribed_dofs=tuple(range(6)), n_tstep=N_TSTEP)
    print(f"dynamic {time.time() - t0:.1f} s, {len(rec['i'])} case_solve calls", flush=True)
    hg = np.asarray(dyn.structure.hg, float)
    last = {k: np.asarray(getattr(dyn.aero, k)[0], float) for k in ("gamma_b", "gamma_w", "zeta_w")}
    OUT.parent.mkdir(exist_ok=True)
    np.savez_compressed(
        OUT, dims=np.array([M, n, M_STAR]), n_tstep=N_TSTEP, dt=dt, u_inf=U_INF, rho=RHO, gust_length=GUST_LENGTH,
        gust_amplitude=GUST_AMP, gust_x0=GUST_X0, zeta_b0=np.asarray(uvlm.zeta_b0[0], float),
        hg0=np.asarray(beam.hg0, float), mirror_point=np.zeros(3), mirror_normal=np.array((0.0, 1.0, 0.0)),
        include_unsteady_force=bool(uvlm.include_unsteady_force), kernel="cutoff", r_cut=R_CORE,
        **{f"init_{k}": v for k, v in init.items()},
        rec_i=np.array(rec["i"]), rec_hg_n=np.stack(rec["hg_n"]), rec_hg_nm1=np.stack(rec["hg_nm1"]),
        rec_hg_dot_n=np.stack(rec["hg_dot_n"]), rec_f=np.stack(rec["f"]),
        beam_hg=hg, tip_z=hg[:, -1, 2, 3], **{f"dyn_{k}": v for k, v in last.items()})
    print("wrote", OUT)


if __name__ == "__main__":
    main()
