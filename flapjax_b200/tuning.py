"""Autotuning of the Biot-Savart sum launches (fj_autotune_vind).

A sum of n_targets points over a stream of filament elements runs as target tiles x
splits CTAs.  ``autotune`` times candidate split counts, and for the FP32 sums both tile
shapes (two or four targets per thread), for given shapes on the device and publishes the
fastest in the library's immutable table, which every later launch of
that (precision, log2 targets, log2 stream length) bucket uses; ``step_shapes`` lists the
three sums of one UVLM time step of a case (wake RHS, forces, free-wake convection,
aero/uvlm.py:912-941, 961-983, 1023-1033).  ``save``/``load`` carry a table to another
process.
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from . import _lib


def step_shapes(m: int, n: int, m_star: int, free_wake: bool):
    """(n_targets, n_elem) of the sums in one time step of an m x n wing with m_star wake
    rows: the wake RHS at the collocation points, the forces at the filament midpoints
    (bound + wake streams), and the free-wake convection at the wake vertices."""
    bound = 2 * (m + 1) * (n + 1)
    wake = 2 * (m_star + 1) * (n + 1)
    force_pts = m * (n + 1) + (m + 1) * n
    shapes = [(m * n, wake), (force_pts, bound + wake)]
    if free_wake:
        shapes.append(((m_star + 1) * (n + 1), bound + wake))
    return [s for s in shapes if s[0] > 0 and s[1] > 0]


def autotune(shapes, precision="mixed", kernel=None, r_cut=0.0, device=None):
    """Tune the split of each (n_targets, n_elem) shape; returns one dict per shape with the
    chosen split, the wave-filling rule's split and their times (ms)."""
    import torch

    prec = _lib.FJ_PREC_MIXED if precision == "mixed" else _lib.FJ_PREC_FP64
    kern = _lib.FJ_KERNEL_EPSILON if kernel is None else kernel
    k = len(shapes)
    nt = (C.c_int64 * k)(*[int(s[0]) for s in shapes])
    ne = (C.c_int64 * k)(*[int(s[1]) for s in shapes])
    nbytes = C.c_size_t()
    _lib.call("fj_autotune_vind_workspace_size", prec, nt, ne, k, C.byref(nbytes))
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=dev)
    chosen, heur = (C.c_int * k)(), (C.c_int * k)()
    cms, hms = (C.c_double * k)(), (C.c_double * k)()
    _lib.call("fj_autotune_vind", prec, kern, float(r_cut), nt, ne, k, chosen, heur, cms, hms, ws.data_ptr(),
              ws.numel(), torch.cuda.current_stream(dev).cuda_stream)
    return [{"n_targets": int(nt[i]), "n_elem": int(ne[i]), "split": chosen[i] & 0xFFF,
             "targets_per_thread": 4 if chosen[i] & 0x1000 else 2, "rule_split": heur[i], "ms": cms[i],
             "rule_ms": hms[i]} for i in range(k)]


def table() -> np.ndarray:
    """The published table (int16 entries, 0 = not tuned)."""
    n = C.c_int()
    _lib.call("fj_autotune_table_size", C.byref(n))
    out = np.zeros(n.value, dtype=np.int16)
    _lib.call("fj_autotune_get", out.ctypes.data, n.value)
    return out


def set_table(entries) -> None:
    """Publish a table (None drops it: every launch uses the wave-filling rule)."""
    if entries is None:
        _lib.call("fj_autotune_set", None, 0)
        return
    arr = np.ascontiguousarray(entries, dtype=np.int16)
    _lib.call("fj_autotune_set", arr.ctypes.data, arr.size)


def save(path) -> None:
    t = table()
    nz = np.nonzero(t)[0]
    with open(path, "w") as f:
        json.dump({"size": int(t.size), "entries": {str(int(i)): int(t[i]) for i in nz}}, f)


def load(path) -> None:
    with open(path) as f:
        d = json.load(f)
    t = np.zeros(int(d["size"]), dtype=np.int16)
    for i, v in d["entries"].items():
        t[int(i)] = v
    set_table(t)
