"""``UVLM`` with the reference's call surface (aero/uvlm.py:80-1406), computed by
``libfj_uvlm.so`` on a B200.

Supported: any number of surfaces, the epsilon / cutoff / plain kernels, mirror images,
prescribed and free wakes, the variable wake discretisation ``delta_w``, static (regular
or horseshoe wake) and prescribed-motion dynamic solves, single-step ``case_solve`` for
fluid-structure loops, Constant and OneMinusCosine flows, tabulated strip polars with the
circulation blend.  Not supported (it raises): control surfaces (``grid_func``).

``precision="fp64"`` runs the reference's arithmetic in FP64; ``precision="mixed"`` runs
the Biot-Savart sums in FP32 (FP64 accumulation) and solves with cached FP32 factors
plus FP64 iterative refinement.
"""
from __future__ import annotations

from collections.abc import Sequence

import numpy as np

from . import _lib
from .data_structures import AeroCase, ArrayList, GridDiscretisation
from .flowfields import FlowField
from .kernels import resolve
from .polars import pack_surface, tabulate
from .runtime import DeviceCase, SurfaceLayout

HORSESHOE_LENGTH = 1e3  # utils/constants.py:13

_PREC = {"fp64": _lib.FJ_PREC_FP64, "mixed": _lib.FJ_PREC_MIXED}


def check_arr_shape(arr, expected_shape, name):
    """Shape check with the reference's message (algebra/array_utils.py:17-40)."""
    actual = np.shape(arr)
    if len(actual) == len(expected_shape) and all(e is None or a == e for a, e in zip(actual, expected_shape)):
        return
    message = f"Expected shape {expected_shape}, but got shape {actual}."
    if name is not None:
        message += f"Issue with input '{name}'"
    raise ValueError(message)


def make_rectangular_grid(m: int, n: int, chord: float, ea: float) -> np.ndarray:
    """``make_rectangular_grid`` aero/utils.py:23-36."""
    grid = np.zeros((m + 1, n + 1, 3))
    grid[..., 0] = (np.linspace(0.0, chord, m + 1) - ea * chord)[:, None]
    return grid


def _se3_apply(hg, x):
    return np.einsum("...ij,...j->...i", hg[..., :3, :3], x) + hg[..., :3, 3]


def _neighbour_average(arr, axes):
    for ax in (axes,) if isinstance(axes, int) else axes:
        i1 = [slice(None)] * arr.ndim
        i2 = [slice(None)] * arr.ndim
        i1[ax] = slice(None, -1)
        i2[ax] = slice(1, None)
        arr = 0.5 * (arr[tuple(i1)] + arr[tuple(i2)])
    return arr


def _surf_nc(zeta):
    d1 = zeta[1:, 1:, :] - zeta[:-1, :-1, :]
    d2 = zeta[1:, :-1, :] - zeta[:-1, 1:, :]
    return np.cross(d1, d2)


class UVLM:
    """Unsteady vortex lattice method over any number of lifting surfaces."""

    def __init__(self, grid_shapes: Sequence, dof_mapping, variable_wake_disc: bool = False, mirror_point=None,
                 mirror_normal=None, kernel=None, grid_func=None, free_wake: bool = False,
                 gamma_dot_relaxation: float = 0.7, include_unsteady_force: bool = True, batch_size: int | None = 64,
                 polars=None, polar_circulation_scale: float = 0.0, precision: str = "fp64", device=None):
        # aero/uvlm.py:211-339
        if isinstance(dof_mapping, np.ndarray):
            dof_list = [dof_mapping]
        elif isinstance(dof_mapping, Sequence):
            dof_list = list(dof_mapping)
        else:
            raise TypeError("Invalid dof mapping type")
        self.n_surf = len(grid_shapes)
        if self.n_surf > _lib.FJ_MAX_SURF:
            raise ValueError(f"at most {_lib.FJ_MAX_SURF} surfaces are supported")
        grid_disc = []
        for grid in grid_shapes:
            if isinstance(grid, GridDiscretisation):
                grid_disc.append(grid)
            elif isinstance(grid, Sequence) or (hasattr(grid, "m") and hasattr(grid, "m_star")):
                if isinstance(grid, Sequence):
                    if len(grid) != 3:
                        raise ValueError("Grid shape tuple must have exactly three elements (m, n, m_star)")
                    grid_disc.append(GridDiscretisation(*[int(v) for v in grid]))
                else:
                    grid_disc.append(GridDiscretisation(int(grid.m), int(grid.n), int(grid.m_star)))
            else:
                raise TypeError("Grid shape must be either a Sequence of three integers or a GridDiscretisation instance")
        self.grid_disc = tuple(grid_disc)
        self.n_bound_panels = tuple(gd.m * gd.n for gd in self.grid_disc)
        self.n_wake_panels = tuple(gd.m_star * gd.n for gd in self.grid_disc)
        if len(dof_list) != self.n_surf:
            raise ValueError(f"Expected {self.n_surf} DOF mapping arrays, got {len(dof_list)}")
        self.dof_mapping = ArrayList()
        for i, map_ in enumerate(dof_list):
            arr = np.asarray(map_)
            if not np.issubdtype(arr.dtype, np.integer):
                raise TypeError("dof_mapping must be an integer array")
            check_arr_shape(arr, (self.grid_disc[i].n + 1,), "grid_disc")
            self.dof_mapping.append(arr.astype(np.int32))
        if grid_func is not None:
            raise NotImplementedError("control surfaces (grid_func) are not part of the CUDA path")
        # uvlm.py:294-303: per surface None or n strip polars (tables on the device)
        if polars is None:
            self.polars = tuple([None] * self.n_surf)
        else:
            if len(polars) != self.n_surf:
                raise ValueError(f"Expected {self.n_surf} polar entries, got {len(polars)}")
            self.polars = tuple(None if p is None else tuple(tabulate(f) for f in p) for p in polars)
        if not 0.0 <= polar_circulation_scale <= 1.0:
            raise ValueError(f"polar_circulation_scale must be in [0, 1], got {polar_circulation_scale}.")
        self.polar_circulation_scale = float(polar_circulation_scale)
        if (mirror_point is None) != (mirror_normal is None):
            raise ValueError("Both mirror_point and mirror_normal must be provided to apply mirroring, or both must be "
                             "None to apply no mirroring.")
        if mirror_point is None:
            self.mirror_point = None
            self.mirror_normal = None
        else:
            self.mirror_point = np.asarray(mirror_point, dtype=np.float64)
            mn = np.asarray(mirror_normal, dtype=np.float64)
            self.mirror_normal = mn / np.linalg.norm(mn)
        self.kernel = resolve(kernel)
        if precision not in _PREC:
            raise ValueError(f"precision must be one of {tuple(_PREC)}")
        if precision == "mixed" and self.kernel.kernel_id == _lib.FJ_KERNEL_PLAIN:
            raise ValueError("the unregularised kernel is only available with precision='fp64'")
        self.precision = precision
        self.variable_wake_disc = variable_wake_disc
        self.free_wake = bool(free_wake)
        self.gamma_dot_relaxation = float(gamma_dot_relaxation)
        self.include_unsteady_force = include_unsteady_force
        self.batch_size = batch_size
        self.device = device
        self.flowfield: FlowField | None = None
        self._dt = None
        self.zeta_b0 = None
        self.hg_ref = None
        self.zeta_b_ref = None
        self.zeta_w_ref = None
        self.delta_w = None
        self._step_case = None
        self._step_key = None
        self._step_factored = False
        self._vind_dev = None

    # ---------------------------------------------------------------------------------
    @property
    def dt(self):
        if self._dt is None:
            raise ValueError("Time step length dt has not been set.")
        return self._dt

    def set_design_variables(self, dt, flowfield: FlowField, zeta_b0, hg0, delta_w=None, reference_cs_angles=None):
        """aero/uvlm.py:387-472."""
        if isinstance(delta_w, np.ndarray):
            dws = [delta_w]
        elif delta_w is None:
            dws = [None] * self.n_surf
        elif isinstance(delta_w, Sequence):
            dws = list(delta_w)
        else:
            raise TypeError("Invalid delta_w type")
        if len(dws) != self.n_surf:
            raise ValueError(f"Expected {self.n_surf} delta_w entries, got {len(dws)}")
        if reference_cs_angles:
            raise NotImplementedError("control surfaces are not part of the CUDA path")
        if isinstance(zeta_b0, np.ndarray):
            zl = [zeta_b0]
        elif isinstance(zeta_b0, Sequence):
            zl = list(zeta_b0)
        else:
            raise TypeError("Invalid zeta_b0 type")
        if len(zl) != self.n_surf:
            raise ValueError(f"Expected {self.n_surf} aerodynamic grid coordinate arrays, got {len(zl)}")
        for i in range(self.n_surf):
            check_arr_shape(zl[i], (self.grid_disc[i].m + 1, self.grid_disc[i].n + 1, 3), "zeta_b0")
        self.zeta_b0 = ArrayList([np.asarray(z, dtype=np.float64) for z in zl])
        hg0 = np.asarray(hg0, dtype=np.float64)
        check_arr_shape(hg0, (None, 4, 4), "hg0")
        self.hg_ref = hg0
        self.zeta_b_ref = self.hg_to_zeta_b(hg0)
        self.flowfield = flowfield
        if isinstance(dt, (float, int, np.floating)) or np.ndim(dt) == 0:
            self._dt = float(dt)
        else:
            raise TypeError("dt must be either a float or an Array scalar")
        self.delta_w = []
        for i, dw in enumerate(dws):
            if dw is None:
                self.delta_w.append(None)
            else:
                dw = np.asarray(dw, dtype=np.float64)
                check_arr_shape(dw, (self.grid_disc[i].m_star,), "delta_w")
                self.delta_w.append(dw)
        self.zeta_w_ref = self.initialise_wake()
        self._step_case = None
        self._step_key = None
        self._step_factored = False

    def hg_to_zeta_b(self, hg_n, cs_ang_n=None) -> ArrayList:
        """aero/uvlm.py:537-560 (host evaluation)."""
        return ArrayList([_se3_apply(np.asarray(hg_n)[self.dof_mapping[i]][None], self.zeta_b0[i])
                          for i in range(self.n_surf)])

    def initialise_wake(self, zeta_b=None) -> ArrayList:
        """aero/uvlm.py:662-689 (host evaluation)."""
        zeta_b = zeta_b if zeta_b is not None else self.zeta_b_ref
        out = ArrayList()
        for i in range(self.n_surf):
            zeta_te = zeta_b[i][-1, :, :]
            dw = self.delta_w[i] if self.delta_w and self.delta_w[i] is not None else (
                np.ones(self.grid_disc[i].m_star) * self.dt * self.flowfield.u_inf_mag)
            grid_s = np.concatenate((np.zeros(1), np.cumsum(dw)))
            out.append(zeta_te[None, :, :] + np.outer(grid_s, self.flowfield.u_inf_dir)[:, None, :])
        return out

    # ---------------------------------------------------------------------------------
    def _config(self, n_tstep: int, n_nodes: int) -> _lib.FjCaseConfig:
        if self.flowfield is None:
            raise ValueError("flowfield has not been set")
        c = _lib.FjCaseConfig()
        c.n_surf = self.n_surf
        for i, gd in enumerate(self.grid_disc):
            c.m[i], c.n[i], c.m_star[i] = gd.m, gd.n, gd.m_star
        c.n_nodes = n_nodes
        c.n_tstep = n_tstep
        c.kernel = self.kernel.kernel_id
        c.r_cut = self.kernel.r_cut
        c.free_wake = int(self.free_wake)
        if self.mirror_point is not None:
            c.mirror = 1
            c.mirror_point[:] = self.mirror_point.tolist()
            c.mirror_normal[:] = self.mirror_normal.tolist()
        c.dt = self.dt
        c.gamma_dot_relaxation = self.gamma_dot_relaxation
        c.flow = self.flowfield.to_c()
        c.precision = _PREC[self.precision]
        for i, dw in enumerate(self.delta_w or []):
            c.variable_wake[i] = int(dw is not None)
        for i, (P, _) in enumerate(self._polar_blocks()):
            c.polar_points[i] = P
        c.polar_circulation_scale = self.polar_circulation_scale
        return c

    def _polar_blocks(self):
        """(points per strip, table block) per surface; (0, None) without polars."""
        return [(0, None) if p is None else pack_surface(p, gd.n) for p, gd in zip(self.polars, self.grid_disc)]

    def _polars_flat(self):
        blocks = [b for P, b in self._polar_blocks() if P > 0]
        return None if not blocks else np.concatenate([b.ravel() for b in blocks])

    def _delta_w_flat(self):
        """Concatenated delta_w of every surface (zeros where a surface is uniform), or
        None when no surface has one."""
        if not self.delta_w or all(d is None for d in self.delta_w):
            return None
        return np.concatenate([np.zeros(g.m_star) if d is None else d for d, g in zip(self.delta_w, self.grid_disc)])

    def _layout(self) -> SurfaceLayout:
        return SurfaceLayout(tuple(g.m for g in self.grid_disc), tuple(g.n for g in self.grid_disc),
                             tuple(g.m_star for g in self.grid_disc))

    def make_device_case(self, n_tstep: int, n_nodes: int | None = None, stream=None) -> DeviceCase:
        """Allocate the device state of an ``n_tstep``-slot case."""
        if self.zeta_b0 is None:
            raise ValueError("zeta_b0 has not been set")
        n_nodes = self.hg_ref.shape[0] if n_nodes is None else n_nodes
        for i, d in enumerate(self.dof_mapping):
            if d.min() < 0 or d.max() >= n_nodes:
                raise ValueError(f"dof_mapping[{i}] refers to nodes outside [0, {n_nodes})")
        zeta0 = np.concatenate([z.ravel() for z in self.zeta_b0])
        dof = np.concatenate([d.ravel() for d in self.dof_mapping])
        return DeviceCase(self._config(n_tstep, n_nodes), self._layout(), zeta0, dof, self.device, stream,
                          delta_w=self._delta_w_flat(), polars=self._polars_flat())

    def _to_case(self, dc: DeviceCase, slots=None, snapshot=False) -> AeroCase:
        h = dc.host_arrays(slots)
        f = {name: dc.split_surfaces(name, h[name]) for name in
             ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
              "f_unsteady", "alpha")}
        if snapshot:
            f = {k: [a[0] for a in v] for k, v in f.items()}
            t, i_ts, ft = h["t"][0], 0, h["force_total"][0]
        else:
            t, i_ts, ft = h["t"], np.arange(h["t"].shape[0]), h["force_total"]
        f["n"] = f.pop("nc")
        return AeroCase(**f, t=t, i_ts=i_ts, force_total=ft, **self._case_meta())

    def _case_meta(self) -> dict:
        """What an AeroCase needs from its solver: the flow, the vertex-column -> node map
        (project_forcing_to_beam) and an FP64 induced-velocity sum with this solver's kernel
        and mirror plane (get_v_ind)."""
        return dict(flowfield=self.flowfield, dof_mapping=self.dof_mapping, induced=self._induced)

    def _induced(self, targets, zetas, gammas):
        if self._vind_dev is None:
            from .adjoint import _Dev

            mirror = None if self.mirror_point is None else (self.mirror_point, self.mirror_normal)
            self._vind_dev = _Dev(self.device, self.kernel.kernel_id, self.kernel.r_cut, mirror)
        lats = [(np.asarray(z, float), np.asarray(g, float)) for z, g in zip(zetas, gammas)]
        return self._vind_dev.vind(np.asarray(targets, float), lats)

    @staticmethod
    def _flat(case_field, idx=None):
        return np.concatenate([(a if idx is None else a[idx]).ravel() for a in case_field])

    # ---------------------------------------------------------------------------------
    def solve_static(self, hg=None, t=0.0, horseshoe: bool = False, cs_ang=None) -> AeroCase:
        """aero/uvlm.py:1286-1333: a snapshot AeroCase."""
        hg = self.hg_ref if hg is None else np.asarray(hg, dtype=np.float64)
        dc = self.make_device_case(1, hg.shape[0])
        dc.set_hg(hg[None])
        dc.solve_static(horseshoe, float(t))
        return self._to_case(dc, snapshot=True)

    def linearise(self, reference: AeroCase, wake_type: str, bound_upwash: bool = True, wake_upwash: bool = True,
                  unsteady_force: bool = True):
        """aero/uvlm.py:356-385: the linearised model about ``reference`` (a steady snapshot,
        e.g. ``solve_static()``), with A, B, C, D assembled on the device."""
        from .linear import LinearUVLM

        return LinearUVLM(self, reference=reference, wake_type=wake_type, bound_upwash=bound_upwash,
                          wake_upwash=wake_upwash, unsteady_force=unsteady_force, device=self.device)

    def reference_configuration(self) -> AeroCase:
        """aero/uvlm.py:1408-1446: the undisturbed snapshot with zero circulation."""
        gds = self.grid_disc
        return AeroCase(
            zeta_b=self.zeta_b_ref, zeta_b_dot=[np.zeros((g.m + 1, g.n + 1, 3)) for g in gds],
            zeta_w=self.zeta_w_ref, c=[_neighbour_average(z, (0, 1)) for z in self.zeta_b_ref],
            n=[_surf_nc(z) for z in self.zeta_b_ref], gamma_b=[np.zeros((g.m, g.n)) for g in gds],
            gamma_b_dot=[np.zeros((g.m, g.n)) for g in gds], gamma_w=[np.zeros((g.m_star, g.n)) for g in gds],
            f_steady=[np.zeros((g.m + 1, g.n + 1, 3)) for g in gds],
            f_unsteady=[np.zeros((g.m + 1, g.n + 1, 3)) for g in gds], alpha=[np.zeros((g.n,)) for g in gds],
            t=0.0, i_ts=-1, force_total=np.zeros(3), **self._case_meta())

    def _check_motion(self, hg_t, hg_dot_t):
        check_arr_shape(hg_t, (None, None, 4, 4), "hg_n")
        if np.shape(hg_t) != np.shape(hg_dot_t):
            raise ValueError(f"hg_dot_n must have the same shape as hg_n, got {np.shape(hg_dot_t)} vs {np.shape(hg_t)}")

    def load_initial(self, dc: DeviceCase, init_case: AeroCase):
        """Copy a snapshot into slot 0 of a device case."""
        vals = {"zeta_b": self._flat(init_case.zeta_b), "zeta_b_dot": self._flat(init_case.zeta_b_dot),
                "zeta_w": self._flat(init_case.zeta_w), "c": self._flat(init_case.c), "nc": self._flat(init_case.nc),
                "gamma_b": self._flat(init_case.gamma_b), "gamma_b_dot": self._flat(init_case.gamma_b_dot),
                "gamma_w": self._flat(init_case.gamma_w), "f_steady": self._flat(init_case.f_steady),
                "f_unsteady": self._flat(init_case.f_unsteady), "alpha": self._flat(init_case.alpha)}
        ft = init_case.force_total
        if ft is None:  # a snapshot built elsewhere: recompute the sum of vertex forces
            ft = sum(np.asarray(fs).reshape(-1, 3).sum(0) + np.asarray(fu).reshape(-1, 3).sum(0)
                     for fs, fu in zip(init_case.f_steady, init_case.f_unsteady))
        dc.load_slot(0, vals, float(np.asarray(init_case.t)), ft)

    def solve_prescribed_dynamic(self, init_case: AeroCase, hg_t, hg_dot_t, cs_ang_t=None, cs_vel_t=None) -> AeroCase:
        """aero/uvlm.py:1335-1406: a batched AeroCase of ``hg_t.shape[0]`` slots."""
        if cs_ang_t or cs_vel_t:
            raise NotImplementedError("control surfaces are not part of the CUDA path")
        hg_t = np.asarray(hg_t, dtype=np.float64)
        hg_dot_t = np.asarray(hg_dot_t, dtype=np.float64)
        self._check_motion(hg_t, hg_dot_t)
        if init_case.is_batched:
            raise TypeError("to_dynamic only supported for snapshot AeroCase")
        n_tstep = hg_t.shape[0]
        dc = self.make_device_case(n_tstep, hg_t.shape[1])
        self.load_initial(dc, init_case)
        dc.set_hg(hg_t, hg_dot_t)
        dc.solve_dynamic(1, n_tstep)
        return self._to_case(dc)

    def case_solve(self, case: AeroCase, i_ts: int, hg_n, hg_nm1, hg_dot_n, static: bool, horseshoe: bool,
                   cs_ang_n=None, cs_ang_nm1=None, cs_vel_n=None) -> AeroCase:
        """aero/uvlm.py:1119-1215: solve slot ``i_ts`` of a batched case in place."""
        if cs_ang_n or cs_ang_nm1 or cs_vel_n:
            raise NotImplementedError("control surfaces are not part of the CUDA path")
        if static:
            snap = self.solve_static(hg=hg_n, t=float(case.t[i_ts]), horseshoe=horseshoe)
            for k in ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_w", "f_steady", "alpha"):
                case.set_arraylist_at_ts(k, getattr(snap, k), i_ts)
            return case
        hg_n = np.asarray(hg_n, dtype=np.float64)
        hg_nm1 = np.asarray(hg_nm1, dtype=np.float64)
        n_nodes = hg_n.shape[0]
        dc = self._step_case
        if dc is None or dc.cfg.n_nodes != n_nodes:
            dc = self._step_case = self.make_device_case(2, n_nodes)
            self._step_key = None
            self._step_factored = False
        prev = case[i_ts - 1]
        # A fluid-structure loop re-solves slot i_ts with new frames hg_n from the same
        # converged slot i_ts-1: the free-wake convection (which depends on slot i_ts-1 and
        # hg_nm1 only, uvlm.py:912-941) is then taken from the previous call.
        key = (i_ts, hg_nm1, [np.asarray(a) for a in prev.gamma_b], [np.asarray(a) for a in prev.gamma_w],
               [np.asarray(a) for a in prev.zeta_w])
        old = self._step_key
        reuse_conv = bool(self.free_wake and old is not None and old[0] == i_ts and np.array_equal(old[1], hg_nm1)
                          and all(np.array_equal(a, b) for x, y in zip(old[2:], key[2:]) for a, b in zip(x, y)))
        self.load_initial(dc, prev)
        dc.set_hg(np.stack([hg_nm1, hg_n]), np.stack([np.zeros_like(hg_n), np.asarray(hg_dot_n, dtype=np.float64)]))
        # mixed: the FP32 factors of the previous call serve as the refinement's
        # preconditioner; the residual check refactorises if they no longer do
        dc.solve_dynamic(1, 2, reuse_factors=self._step_factored, reuse_convection=reuse_conv)
        self._step_factored = self.precision == "mixed"
        self._step_key = (key[0], key[1].copy(), [a.copy() for a in key[2]], [a.copy() for a in key[3]],
                          [a.copy() for a in key[4]])
        out = self._to_case(dc, slots=slice(1, 2))
        for k in ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
                  "f_unsteady", "alpha"):
            case.set_arraylist_at_ts(k, [a[0] for a in getattr(out, k)], i_ts)
        case.t[i_ts] = out.t[0]
        if case.force_total is not None:
            case.force_total[i_ts] = out.force_total[0]
        return case
