"""Device-side state of one UVLM case and the calls that advance it.

PyTorch provides device memory and the stream; every computation is a call into
``libfj_uvlm.so``.  Arrays are time-major with surfaces concatenated inside each slot
(the layout ``include/fj_uvlm.h`` documents for ``fj_case_buffers``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib


def device_of(device):
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("flapjax_b200 needs a CUDA device (sm_100a); there is no CPU fallback")
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device(device)


@dataclass(frozen=True)
class SurfaceLayout:
    """Per-surface block sizes inside one time slot."""

    m: tuple
    n: tuple
    m_star: tuple

    @property
    def n_surf(self):
        return len(self.m)

    def _blocks(self, f):
        out, off = [], 0
        for i in range(self.n_surf):
            size = f(self.m[i], self.n[i], self.m_star[i])
            out.append((off, size))
            off += size
        return out, off

    def zeta_b(self):
        return self._blocks(lambda m, n, ms: (m + 1) * (n + 1) * 3)

    def zeta_w(self):
        return self._blocks(lambda m, n, ms: (ms + 1) * (n + 1) * 3)

    def panels(self, comp=1):
        return self._blocks(lambda m, n, ms: m * n * comp)

    def gamma_w(self):
        return self._blocks(lambda m, n, ms: ms * n)

    def strips(self):
        return self._blocks(lambda m, n, ms: n)

    def shapes(self, field, i):
        m, n, ms = self.m[i], self.n[i], self.m_star[i]
        return {
            "zeta_b": (m + 1, n + 1, 3), "zeta_b_dot": (m + 1, n + 1, 3), "zeta_w": (ms + 1, n + 1, 3),
            "c": (m, n, 3), "nc": (m, n, 3), "gamma_b": (m, n), "gamma_b_dot": (m, n), "gamma_w": (ms, n),
            "f_steady": (m + 1, n + 1, 3), "f_unsteady": (m + 1, n + 1, 3), "alpha": (n,),
        }[field]

    def blocks(self, field):
        return {
            "zeta_b": self.zeta_b, "zeta_b_dot": self.zeta_b, "zeta_w": self.zeta_w,
            "c": lambda: self.panels(3), "nc": lambda: self.panels(3), "gamma_b": self.panels,
            "gamma_b_dot": self.panels, "gamma_w": self.gamma_w, "f_steady": self.zeta_b,
            "f_unsteady": self.zeta_b, "alpha": self.strips,
        }[field]()


FIELDS = ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
          "f_unsteady", "alpha")


class DeviceCase:
    """Outputs, inputs and workspace of one case on one GPU."""

    def __init__(self, cfg: _lib.FjCaseConfig, layout: SurfaceLayout, zeta_b0: np.ndarray, dof_mapping: np.ndarray,
                 device=None, stream=None, delta_w: np.ndarray | None = None, polars: np.ndarray | None = None):
        import torch

        self.torch = torch
        self.dev = device_of(device)
        self.cfg = cfg
        self.layout = layout
        self.n_tstep = cfg.n_tstep
        self.stream = stream
        f64 = dict(dtype=torch.float64, device=self.dev)
        self.t = torch.zeros(self.n_tstep, **f64)
        self.arrays = {}
        for name in FIELDS:
            _, total = layout.blocks(name)
            self.arrays[name] = torch.zeros((self.n_tstep, total), **f64)
        self.force_total = torch.zeros((self.n_tstep, 3), **f64)
        self.zeta_b0 = torch.from_numpy(np.ascontiguousarray(zeta_b0, dtype=np.float64)).to(self.dev)
        self.dof = torch.from_numpy(np.ascontiguousarray(dof_mapping, dtype=np.int32)).to(self.dev)
        self.delta_w = None if delta_w is None else torch.from_numpy(
            np.ascontiguousarray(delta_w, dtype=np.float64)).to(self.dev)
        self.polars = None if polars is None else torch.from_numpy(
            np.ascontiguousarray(polars, dtype=np.float64)).to(self.dev)
        self.hg_t = torch.zeros((self.n_tstep, cfg.n_nodes, 4, 4), **f64)
        self.hg_dot_t = torch.zeros((self.n_tstep, cfg.n_nodes, 4, 4), **f64)
        nbytes = C.c_size_t()
        _lib.call("fj_case_workspace_size", C.byref(cfg), C.byref(nbytes))
        self.ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.dev)
        self._bufs = self._make_bufs()

    def _make_bufs(self) -> _lib.FjCaseBuffers:
        b = _lib.FjCaseBuffers()
        b.d_zeta_b0 = self.zeta_b0.data_ptr()
        b.d_dof_mapping = self.dof.data_ptr()
        b.d_hg_t = self.hg_t.data_ptr()
        b.d_hg_dot_t = self.hg_dot_t.data_ptr()
        b.d_delta_w = None if self.delta_w is None else self.delta_w.data_ptr()
        b.d_t = self.t.data_ptr()
        for name in FIELDS:
            setattr(b, "d_" + name, self.arrays[name].data_ptr())
        b.d_force_total = self.force_total.data_ptr()
        b.d_polars = None if self.polars is None else self.polars.data_ptr()
        return b

    def _stream(self):
        if self.stream is not None:
            return self.stream.cuda_stream
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    # -- inputs -----------------------------------------------------------------------
    def set_hg(self, hg_t, hg_dot_t=None, non_blocking=False):
        """Copy node frames into the first len(hg_t) slots (host or device arrays)."""
        src = self.torch.as_tensor(hg_t, dtype=self.torch.float64)
        self.hg_t[: src.shape[0]].copy_(src, non_blocking=non_blocking)
        if hg_dot_t is not None:
            srd = self.torch.as_tensor(hg_dot_t, dtype=self.torch.float64)
            self.hg_dot_t[: srd.shape[0]].copy_(srd, non_blocking=non_blocking)

    def load_slot(self, slot: int, values: dict, t: float, force_total=None):
        """Write one solution slot from host arrays (per-field, surfaces concatenated)."""
        for name, arr in values.items():
            self.arrays[name][slot].copy_(self.torch.as_tensor(np.ascontiguousarray(arr).ravel()))
        self.t[slot] = float(t)
        if force_total is not None:
            self.force_total[slot].copy_(self.torch.as_tensor(np.asarray(force_total, dtype=np.float64)))

    def copy_slot_from(self, other: "DeviceCase", slot: int):
        """Device-to-device copy of one solution slot from a case of the same layout."""
        for name, a in self.arrays.items():
            a[slot].copy_(other.arrays[name][slot])
        self.t[slot].copy_(other.t[slot])
        self.force_total[slot].copy_(other.force_total[slot])

    # -- compute ----------------------------------------------------------------------
    def solve_static(self, horseshoe: bool, t0: float):
        _lib.call("fj_solve_static", C.byref(self.cfg), C.byref(self._bufs), int(horseshoe), float(t0),
                  self.ws.data_ptr(), self.ws.numel(), self._stream())

    def solve_dynamic(self, i_first: int, i_last: int, reuse_factors: bool = False, graph: bool = True,
                      reuse_convection: bool = False):
        """Steps i_first..i_last-1.  ``reuse_factors``: keep the mixed path's cached
        factors from the previous call on this case.  ``graph``: replay runs of steps from
        one captured CUDA graph (False: launch every step directly; same results).
        ``reuse_convection``: the previous call solved slot i_first from the same slot
        i_first-1 and frames hg_t[i_first-1] (a fluid-structure iteration), so its free-wake
        convection velocities are taken instead of recomputed."""
        flags = ((_lib.FJ_REUSE_FACTORS if reuse_factors else 0) | (0 if graph else _lib.FJ_NO_GRAPH)
                 | (_lib.FJ_REUSE_CONVECTION if reuse_convection else 0))
        _lib.call("fj_solve_prescribed_dynamic", C.byref(self.cfg), C.byref(self._bufs), int(i_first), int(i_last),
                  flags, self.ws.data_ptr(), self.ws.numel(), self._stream())

    def copy_factors(self, lu, piv):
        """Copy the FP64 getrf factors and pivots of the last solved step into the
        device tensors ``lu`` (nb x nb, float64) and ``piv`` (nb, int32)."""
        _lib.call("fj_case_factors_copy", C.byref(self.cfg), self.ws.data_ptr(), self.ws.numel(), lu.data_ptr(),
                  piv.data_ptr(), self._stream())

    # -- outputs ----------------------------------------------------------------------
    def host_arrays(self, slots=None):
        """Numpy copies {field: (n_slots, total)} of the given slots (default all)."""
        sl = slice(None) if slots is None else slots
        out = {name: a[sl].cpu().numpy() for name, a in self.arrays.items()}
        out["t"] = self.t[sl].cpu().numpy()
        out["force_total"] = self.force_total[sl].cpu().numpy()
        return out

    def split_surfaces(self, field, flat):
        """(n_slots, total) -> list over surfaces of (n_slots, *shape)."""
        blocks, _ = self.layout.blocks(field)
        return [flat[:, off:off + size].reshape((flat.shape[0],) + self.layout.shapes(field, i))
                for i, (off, size) in enumerate(blocks)]
