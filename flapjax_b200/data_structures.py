"""Host containers mirroring the reference's aero pytrees.

``GridDiscretisation`` (aero/data_structures.py:29-40), ``ArrayList``
(algebra/array_utils.py:139) and ``AeroCase`` (aero/data_structures.py:43-615) with the
same field names and per-surface layouts: a snapshot holds ``(m+1, n+1, 3)`` lattices and
``(m, n)`` circulations per surface; a batched case adds a leading time axis.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class GridDiscretisation:
    """Chordwise, spanwise and wake panel counts of one surface."""

    m: int
    n: int
    m_star: int


class ArrayList(list):
    """A list of per-surface arrays."""

    def index_all(self, *idx):
        return ArrayList([a[idx] for a in self])

    def copy(self):
        return ArrayList([np.array(a, copy=True) for a in self])


_FIELDS = ("zeta_b", "zeta_b_dot", "zeta_w", "c", "nc", "gamma_b", "gamma_b_dot", "gamma_w", "f_steady",
           "f_unsteady", "alpha")


class AeroCase:
    """UVLM solution over one (snapshot) or many (batched) time steps.

    Fields as the reference: ``zeta_b, zeta_b_dot, zeta_w, c, nc, gamma_b, gamma_b_dot,
    gamma_w, f_steady, f_unsteady, alpha`` (ArrayLists), ``t`` and ``i_ts``.  ``force_total``
    (per slot, sum over every vertex of ``f_steady + f_unsteady``) is an addition.
    """

    def __init__(self, zeta_b, zeta_b_dot, zeta_w, c, n, gamma_b, gamma_b_dot, gamma_w, f_steady, f_unsteady, alpha,
                 t, i_ts, force_total=None, **meta):
        self.zeta_b = ArrayList(zeta_b)
        self.zeta_b_dot = ArrayList(zeta_b_dot)
        self.zeta_w = ArrayList(zeta_w)
        self.c = ArrayList(c)
        self.nc = ArrayList(n)
        self.gamma_b = ArrayList(gamma_b)
        self.gamma_b_dot = ArrayList(gamma_b_dot)
        self.gamma_w = ArrayList(gamma_w)
        self.f_steady = ArrayList(f_steady)
        self.f_unsteady = ArrayList(f_unsteady)
        self.alpha = ArrayList(alpha)
        self.t = np.asarray(t, dtype=np.float64)
        self.i_ts = i_ts
        self.force_total = None if force_total is None else np.asarray(force_total)
        self.meta = meta

    @property
    def is_batched(self) -> bool:
        return self.gamma_b[0].ndim == 3  # aero/data_structures.py:161-164

    @property
    def n_tstep(self) -> int:
        if not self.is_batched:
            raise TypeError("n_tstep only defined for a batched AeroCase")
        return self.gamma_b[0].shape[0]

    def _fields(self):
        return {k: getattr(self, k) for k in _FIELDS}

    def __getitem__(self, idx: int) -> "AeroCase":
        """Snapshot at time index ``idx`` (aero/data_structures.py:533-568)."""
        if not self.is_batched:
            raise TypeError("__getitem__ only supported for batched AeroCase")
        f = {k: [a[idx] for a in v] for k, v in self._fields().items()}
        f["n"] = f.pop("nc")
        ft = None if self.force_total is None else self.force_total[idx]
        return AeroCase(**f, t=self.t[idx], i_ts=idx, force_total=ft, **self.meta)

    def to_dynamic(self, i_ts: int, n_tstep: int) -> "AeroCase":
        """Expand a snapshot into ``n_tstep`` zero-filled slots with the snapshot at
        ``i_ts`` (aero/data_structures.py:570-610)."""
        if self.is_batched:
            raise TypeError("to_dynamic only supported for snapshot AeroCase")
        f = {}
        for k, v in self._fields().items():
            out = []
            for a in v:
                z = np.zeros((n_tstep,) + np.shape(a))
                z[i_ts] = a
                out.append(z)
            f[k] = out
        f["n"] = f.pop("nc")
        t = np.zeros(n_tstep)
        t[i_ts] = self.t
        ft = None
        if self.force_total is not None:
            ft = np.zeros((n_tstep, 3))
            ft[i_ts] = self.force_total
        return AeroCase(**f, t=t, i_ts=np.arange(n_tstep), force_total=ft, **self.meta)

    def set_arraylist_at_ts(self, attr: str, values, i_ts: int) -> None:
        if not self.is_batched:
            raise TypeError("set_arraylist_at_ts only supported for batched AeroCase")
        arr = getattr(self, attr)
        for i, val in enumerate(values):
            arr[i][i_ts] = val
